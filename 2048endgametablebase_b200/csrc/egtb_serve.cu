// Serving loop of libegtb_gpu: books resident in device memory, a scheduler
// thread that batches incoming position queries of any size into in-flight
// slots (continuous batching), and a replay harness for latency measurement.
//
// A slot is one batch on its own CUDA stream with pinned input/output
// buffers and a completion event. The scheduler retires finished slots,
// copies their answers to the requests' buffers, and fills every free slot
// with queued requests in arrival order while they fit in the slot's
// position capacity (memory-based admission). Requests that arrive while
// slots are on the GPU wait in the queue and join the next free slot, so up
// to `slots` batches overlap on the device (copies and kernels of different
// slots run concurrently). Requests whose buffers lie in memory registered
// with the server skip the staging copies: the slot passes the kernel a list
// of {positions, answers} device addresses and the kernel works in place.
//
// The reference answers one position per call from files
// (ClassicBookReader.move_on_dic, native_core/src/ReaderRuntime.cpp:1050-1067);
// every answer here is that call's answer with last_op = 0, as float32.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "egtb_host.h"

// from egtb_book.cu
namespace egtb {
int book_device(const egtb_book *b);
void book_lookup_requests(egtb_book *b, const ServeReq *d_reqs, int n_req, unsigned long long total, cudaStream_t s);
}  // namespace egtb

namespace egtb {

using Clock = std::chrono::steady_clock;

struct ServeRequest {
    uint64_t ticket = 0;
    int book = 0;
    const uint64_t *pos = nullptr;
    size_t n = 0;
    float *out = nullptr;
    uint8_t *valid = nullptr;
    // direct: every buffer lies in registered memory; the kernel reads and
    // writes it through these device addresses (no staging copies)
    bool direct = false;
    const uint64_t *d_pos = nullptr;
    float *d_out = nullptr;
    uint8_t *d_valid = nullptr;
    Clock::time_point t_submit;
    // latency is measured from here: the submit time, or for a replayed
    // stream the request's scheduled arrival (so time a late driver thread
    // spent behind the schedule counts as queueing)
    Clock::time_point t_arrival;
    double latency_us = 0.0;
    bool done = false;
};

// Caller memory registered with the server (page-locked and mapped).
struct Registered {
    uintptr_t begin, end;
    uintptr_t dev;
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t event = nullptr;
    uint64_t *h_pos = nullptr, *d_pos = nullptr;
    float *h_out = nullptr, *d_out = nullptr;
    uint8_t *h_valid = nullptr, *d_valid = nullptr;
    size_t cap = 0;
    ServeReq *h_reqs = nullptr, *d_reqs = nullptr;  // request lists of the direct requests
    size_t req_cap = 0;
    bool busy = false;
    std::vector<ServeRequest *> reqs;
    std::vector<size_t> at;  // position offset of each staged request in the slot
};

}  // namespace egtb

struct egtb_server {
    int device = 0;
    std::vector<egtb_book *> books;
    std::vector<egtb::Slot> slots;
    size_t max_per_batch = 0;  // 0: no limit; 1: one request per launch (the unbatched baseline)
    std::mutex mu;
    std::condition_variable cv_done;
    std::deque<egtb::ServeRequest *> queue;
    std::unordered_map<uint64_t, std::unique_ptr<egtb::ServeRequest>> live;
    std::vector<egtb::Registered> registered;
    uint64_t next_ticket = 1;
    std::atomic<bool> stop{false};
    std::thread worker;
    std::string error;
    // statistics
    uint64_t n_requests = 0, n_positions = 0, n_batches = 0, n_launches = 0;
};

namespace egtb {

static void serve_loop(egtb_server *S) {
    try {
        EGTB_CUDA(cudaSetDevice(S->device));
        std::vector<ServeRequest *> finished;
        while (!S->stop.load(std::memory_order_relaxed)) {
            bool worked = false;
            // 1. retire finished slots
            for (auto &sl : S->slots) {
                if (!sl.busy) continue;
                const cudaError_t q = cudaEventQuery(sl.event);
                if (q == cudaErrorNotReady) continue;
                EGTB_CUDA(q);
                const auto now = Clock::now();
                for (size_t r = 0; r < sl.reqs.size(); ++r) {
                    ServeRequest *rq = sl.reqs[r];
                    if (!rq->direct) {
                        std::memcpy(rq->out, sl.h_out + 4 * sl.at[r], rq->n * 4 * sizeof(float));
                        if (rq->valid) std::memcpy(rq->valid, sl.h_valid + sl.at[r], rq->n);
                    }
                    rq->latency_us = std::chrono::duration<double, std::micro>(now - rq->t_arrival).count();
                    finished.push_back(rq);
                }
                sl.reqs.clear();
                sl.at.clear();
                sl.busy = false;
                worked = true;
            }
            if (!finished.empty()) {
                {
                    std::lock_guard<std::mutex> lk(S->mu);
                    for (auto *rq : finished) rq->done = true;
                }
                S->cv_done.notify_all();
                finished.clear();
            }
            // 2. admit queued requests into every free slot
            for (auto &sl : S->slots) {
                if (sl.busy) continue;
                std::vector<ServeRequest *> take;
                {
                    std::lock_guard<std::mutex> lk(S->mu);
                    size_t used = 0;
                    size_t n_direct = 0;
                    while (!S->queue.empty()) {
                        ServeRequest *rq = S->queue.front();
                        if (used + rq->n > sl.cap) break;  // does not fit: it opens the next slot
                        if (S->max_per_batch && take.size() >= S->max_per_batch) break;
                        if (rq->direct && n_direct + S->books.size() + 1 > sl.req_cap) break;
                        take.push_back(rq);
                        used += rq->n;
                        n_direct += rq->direct;
                        S->queue.pop_front();
                    }
                }
                if (take.empty()) break;
                // group by book so every book gets one contiguous launch per kind
                std::stable_sort(take.begin(), take.end(), [](const ServeRequest *a, const ServeRequest *b) {
                    return a->book != b->book ? a->book < b->book : a->direct < b->direct;
                });
                size_t used = 0, nd = 0;
                std::vector<std::pair<size_t, size_t>> groups;  // staged: [first, last) of take per book
                std::vector<std::pair<int, std::pair<size_t, size_t>>> dgroups;  // direct: book, entries
                for (size_t i = 0; i < take.size();) {
                    size_t j = i;
                    const int book = take[i]->book;
                    const bool direct = take[i]->direct;
                    while (j < take.size() && take[j]->book == book && take[j]->direct == direct) ++j;
                    if (!direct) {
                        groups.push_back({i, j});
                        for (size_t k = i; k < j; ++k) {
                            ServeRequest *rq = take[k];
                            sl.reqs.push_back(rq);
                            sl.at.push_back(used);
                            std::memcpy(sl.h_pos + used, rq->pos, rq->n * sizeof(uint64_t));
                            used += rq->n;
                        }
                    } else {
                        const size_t first = nd;
                        unsigned long long at = 0;
                        for (size_t k = i; k < j; ++k) {
                            ServeRequest *rq = take[k];
                            sl.reqs.push_back(rq);
                            sl.at.push_back(0);
                            sl.h_reqs[nd++] = ServeReq{rq->d_pos, rq->d_out, rq->d_valid, at};
                            at += rq->n;
                        }
                        sl.h_reqs[nd++] = ServeReq{nullptr, nullptr, nullptr, at};  // closes the list
                        dgroups.push_back({book, {first, j - i}});
                        S->n_positions += at;
                    }
                    i = j;
                }
                if (nd)
                    EGTB_CUDA(cudaMemcpyAsync(sl.d_reqs, sl.h_reqs, nd * sizeof(ServeReq), cudaMemcpyHostToDevice,
                                              sl.stream));
                for (const auto &g : dgroups) {
                    book_lookup_requests(S->books[g.first], sl.d_reqs + g.second.first, (int)g.second.second,
                                         sl.h_reqs[g.second.first + g.second.second].at, sl.stream);
                    ++S->n_launches;
                }
                if (used) {
                    EGTB_CUDA(cudaMemcpyAsync(sl.d_pos, sl.h_pos, used * sizeof(uint64_t), cudaMemcpyHostToDevice,
                                              sl.stream));
                    size_t a = 0;
                    for (const auto &g : groups) {
                        size_t cnt = 0;
                        for (size_t k = g.first; k < g.second; ++k) cnt += take[k]->n;
                        if (egtb_book_lookup_device(S->books[take[g.first]->book], sl.d_pos + a, cnt, 0,
                                                    sl.d_out + 4 * a, sl.d_valid + a, sl.stream) != EGTB_OK)
                            throw Error(EGTB_ERR_CUDA, "book lookup launch failed");
                        ++S->n_launches;
                        a += cnt;
                    }
                    EGTB_CUDA(cudaMemcpyAsync(sl.h_out, sl.d_out, used * 4 * sizeof(float), cudaMemcpyDeviceToHost,
                                              sl.stream));
                    EGTB_CUDA(cudaMemcpyAsync(sl.h_valid, sl.d_valid, used, cudaMemcpyDeviceToHost, sl.stream));
                }
                EGTB_CUDA(cudaEventRecord(sl.event, sl.stream));
                sl.busy = true;
                ++S->n_batches;
                S->n_positions += used;
                S->n_requests += take.size();
                worked = true;
            }
            if (!worked) std::this_thread::yield();
        }
    } catch (const std::exception &e) {
        std::lock_guard<std::mutex> lk(S->mu);
        S->error = e.what();
        S->stop = true;
    }
    S->cv_done.notify_all();
}

}  // namespace egtb

using namespace egtb;

extern "C" int egtb_serve_start(egtb_book *const *books, int32_t n_books, int32_t slots, uint64_t slot_positions,
                                int32_t max_requests_per_batch, egtb_server **out) {
    return guarded([&] {
        if (!books || n_books <= 0 || !out) throw Error(EGTB_ERR_ARG, "books and out are required");
        if (slots <= 0 || slots > 64) throw Error(EGTB_ERR_ARG, "slots must be 1..64");
        if (slot_positions < 4096) throw Error(EGTB_ERR_ARG, "slot_positions must hold one full request (4096)");
        for (int i = 0; i < n_books; ++i)
            if (!books[i]) throw Error(EGTB_ERR_ARG, "NULL book");
        auto S = std::make_unique<egtb_server>();
        S->device = book_device(books[0]);
        for (int i = 0; i < n_books; ++i) {
            if (book_device(books[i]) != S->device) throw Error(EGTB_ERR_ARG, "all books must live on one device");
            S->books.push_back(books[i]);
        }
        S->max_per_batch = max_requests_per_batch > 0 ? (size_t)max_requests_per_batch : 0;
        EGTB_CUDA(cudaSetDevice(S->device));
        S->slots.resize(slots);
        for (auto &sl : S->slots) {
            sl.cap = slot_positions;
            EGTB_CUDA(cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking));
            EGTB_CUDA(cudaEventCreateWithFlags(&sl.event, cudaEventDisableTiming));
            EGTB_CUDA(cudaHostAlloc((void **)&sl.h_pos, slot_positions * 8, cudaHostAllocDefault));
            EGTB_CUDA(cudaHostAlloc((void **)&sl.h_out, slot_positions * 16, cudaHostAllocDefault));
            EGTB_CUDA(cudaHostAlloc((void **)&sl.h_valid, slot_positions, cudaHostAllocDefault));
            EGTB_CUDA(cudaMalloc(&sl.d_pos, slot_positions * 8));
            EGTB_CUDA(cudaMalloc(&sl.d_out, slot_positions * 16));
            EGTB_CUDA(cudaMalloc(&sl.d_valid, slot_positions));
            sl.req_cap = std::min<size_t>(slot_positions, 65536) + 2 * S->books.size() + 2;
            EGTB_CUDA(cudaHostAlloc((void **)&sl.h_reqs, sl.req_cap * sizeof(ServeReq), cudaHostAllocDefault));
            EGTB_CUDA(cudaMalloc(&sl.d_reqs, sl.req_cap * sizeof(ServeReq)));
        }
        egtb_server *raw = S.release();
        raw->worker = std::thread(serve_loop, raw);
        *out = raw;
    });
}

namespace egtb {

// egtb_serve_submit with the time its latency is measured from (arrival <= now).
static int serve_submit_at(egtb_server *S, int32_t book, const uint64_t *positions, uint64_t n, float *values4,
                           uint8_t *valid_mask, uint64_t *ticket, const Clock::time_point *arrival) {
    return guarded([&] {
        if (!S || !ticket) throw Error(EGTB_ERR_ARG, "NULL argument");
        if (book < 0 || book >= (int)S->books.size()) throw Error(EGTB_ERR_ARG, "book index out of range");
        if (n == 0 || n > S->slots[0].cap) throw Error(EGTB_ERR_ARG, "request size must be 1..slot_positions");
        if (!positions || !values4) throw Error(EGTB_ERR_ARG, "NULL buffer");
        auto rq = std::make_unique<ServeRequest>();
        rq->book = book;
        rq->pos = positions;
        rq->n = n;
        rq->out = values4;
        rq->valid = valid_mask;
        std::lock_guard<std::mutex> lk(S->mu);
        if (!S->error.empty()) throw Error(EGTB_ERR_CUDA, "server stopped: " + S->error);
        // device address of [p, p + bytes) when it lies in registered memory
        auto mapped = [&](const void *p, size_t bytes) -> uintptr_t {
            const uintptr_t a = (uintptr_t)p;
            for (const auto &r : S->registered)
                if (a >= r.begin && a + bytes <= r.end) return r.dev + (a - r.begin);
            return 0;
        };
        const uintptr_t dp = mapped(positions, n * 8), dout = mapped(values4, n * 16);
        const uintptr_t dv = valid_mask ? mapped(valid_mask, n) : 0;
        if (dp && dout && (dv || !valid_mask)) {
            rq->direct = true;
            rq->d_pos = (const uint64_t *)dp;
            rq->d_out = (float *)dout;
            rq->d_valid = (uint8_t *)dv;
        }
        rq->t_submit = Clock::now();
        rq->t_arrival = arrival ? std::min(*arrival, rq->t_submit) : rq->t_submit;
        rq->ticket = S->next_ticket++;
        *ticket = rq->ticket;
        S->queue.push_back(rq.get());
        S->live.emplace(rq->ticket, std::move(rq));
    });
}

// [a, a + bytes) overlaps [r.begin, r.end)
static bool overlaps(const void *a, size_t bytes, const Registered &r) {
    const uintptr_t x = (uintptr_t)a;
    return a && bytes && x < r.end && x + bytes > r.begin;
}

}  // namespace egtb

extern "C" int egtb_serve_submit(egtb_server *S, int32_t book, const uint64_t *positions, uint64_t n, float *values4,
                                 uint8_t *valid_mask, uint64_t *ticket) {
    return serve_submit_at(S, book, positions, n, values4, valid_mask, ticket, nullptr);
}

extern "C" int egtb_serve_register(egtb_server *S, void *ptr, uint64_t bytes) {
    return guarded([&] {
        if (!S || !ptr || !bytes) throw Error(EGTB_ERR_ARG, "NULL or empty range");
        EGTB_CUDA(cudaSetDevice(S->device));
        EGTB_CUDA(cudaHostRegister(ptr, bytes, cudaHostRegisterMapped | cudaHostRegisterPortable));
        void *dev = nullptr;
        const cudaError_t e = cudaHostGetDevicePointer(&dev, ptr, 0);
        if (e != cudaSuccess) {
            cudaHostUnregister(ptr);
            EGTB_CUDA(e);
        }
        std::lock_guard<std::mutex> lk(S->mu);
        S->registered.push_back(Registered{(uintptr_t)ptr, (uintptr_t)ptr + bytes, (uintptr_t)dev});
    });
}

extern "C" int egtb_serve_unregister(egtb_server *S, void *ptr) {
    return guarded([&] {
        if (!S || !ptr) throw Error(EGTB_ERR_ARG, "NULL argument");
        std::lock_guard<std::mutex> lk(S->mu);
        // a direct request that is not done (queued or on the GPU) reads its
        // positions and writes its answers through the mapped addresses
        for (const auto &q : S->live) {
            const ServeRequest &rq = *q.second;
            if (!rq.direct || rq.done) continue;
            for (const auto &r : S->registered)
                if (r.begin == (uintptr_t)ptr &&
                    (overlaps(rq.pos, rq.n * 8, r) || overlaps(rq.out, rq.n * 16, r) || overlaps(rq.valid, rq.n, r)))
                    throw Error(EGTB_ERR_ARG, "a request in flight uses this range");
        }
        for (size_t i = 0; i < S->registered.size(); ++i)
            if (S->registered[i].begin == (uintptr_t)ptr) {
                EGTB_CUDA(cudaHostUnregister(ptr));
                S->registered.erase(S->registered.begin() + (long)i);
                return;
            }
        throw Error(EGTB_ERR_ARG, "range not registered");
    });
}

extern "C" int egtb_serve_wait(egtb_server *S, uint64_t ticket, int32_t timeout_ms, double *latency_us) {
    return guarded([&] {
        if (!S) throw Error(EGTB_ERR_ARG, "NULL server");
        std::unique_lock<std::mutex> lk(S->mu);
        auto it = S->live.find(ticket);
        if (it == S->live.end()) throw Error(EGTB_ERR_ARG, "unknown ticket");
        ServeRequest *rq = it->second.get();
        const bool ok = S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms < 0 ? 3600000 : timeout_ms),
                                            [&] { return rq->done || !S->error.empty(); });
        if (!S->error.empty()) throw Error(EGTB_ERR_CUDA, "server stopped: " + S->error);
        if (!ok) throw Error(EGTB_ERR_TIMEOUT, "request not answered in time");
        if (latency_us) *latency_us = rq->latency_us;
        S->live.erase(it);
    });
}

extern "C" int egtb_serve_stats(egtb_server *S, uint64_t *requests, uint64_t *positions, uint64_t *batches,
                                uint64_t *launches) {
    return guarded([&] {
        if (!S) throw Error(EGTB_ERR_ARG, "NULL server");
        std::lock_guard<std::mutex> lk(S->mu);
        if (requests) *requests = S->n_requests;
        if (positions) *positions = S->n_positions;
        if (batches) *batches = S->n_batches;
        if (launches) *launches = S->n_launches;
    });
}

extern "C" int egtb_serve_replay(egtb_server *S, const uint64_t *pool, const double *arrival_us, const uint32_t *sizes,
                                 const uint64_t *offsets, const int32_t *books, uint64_t n_req, float *values4,
                                 uint8_t *valid, double *latency_us, double *wall_us) {
    return guarded([&] {
        if (!S || !pool || !arrival_us || !sizes || !offsets || !books || !values4 || !latency_us)
            throw Error(EGTB_ERR_ARG, "NULL argument");
        std::vector<uint64_t> tickets(n_req, 0);
        // the recorded stream's buffers are registered for the run: the kernel
        // reads positions and writes answers in place
        unsigned long long total = 0;
        for (uint64_t i = 0; i < n_req; ++i) total = std::max<unsigned long long>(total, offsets[i] + sizes[i]);
        std::vector<void *> reg;
        auto reg_range = [&](void *p, uint64_t bytes) {
            if (!p || !bytes) return;
            if (egtb_serve_register(S, p, bytes) != EGTB_OK) throw Error(EGTB_ERR_CUDA, "replay: register failed");
            reg.push_back(p);
        };
        struct Unreg {
            egtb_server *S;
            std::vector<void *> &v;
            ~Unreg() {
                for (void *p : v) egtb_serve_unregister(S, p);
            }
        } unreg{S, reg};
        reg_range((void *)pool, total * 8);
        reg_range(values4, total * 16);
        reg_range(valid, total);
        const auto t0 = Clock::now();
        std::atomic<uint64_t> submitted{0};
        std::atomic<bool> failed{false}, halt{false};
        // the driver thread submits every request at its arrival time; each
        // request's latency counts from its scheduled arrival
        std::thread driver([&] {
            for (uint64_t i = 0; i < n_req && !halt.load(std::memory_order_relaxed); ++i) {
                const auto due = t0 + std::chrono::nanoseconds((long long)(arrival_us[i] * 1000.0));
                while (Clock::now() < due) {
                }
                if (serve_submit_at(S, books[i], pool + offsets[i], sizes[i], values4 + 4 * offsets[i],
                                    valid ? valid + offsets[i] : nullptr, &tickets[i], &due) != EGTB_OK) {
                    failed = true;
                    break;
                }
                submitted.store(i + 1, std::memory_order_release);
            }
        });
        uint64_t answered = 0;
        bool timed_out = false;
        for (; answered < n_req; ++answered) {
            while (submitted.load(std::memory_order_acquire) <= answered && !failed) std::this_thread::yield();
            if (submitted.load(std::memory_order_acquire) <= answered) break;
            double lat = 0.0;
            if (egtb_serve_wait(S, tickets[answered], 60000, &lat) != EGTB_OK) {
                timed_out = true;
                break;
            }
            latency_us[answered] = lat;
        }
        if (timed_out) {
            // stop submitting, then give what was submitted a bounded time to
            // finish: the registered ranges are unregistered (by Unreg) only
            // once no request uses them, since the GPU writes answers there
            halt = true;
            driver.join();
            const uint64_t n_sub = submitted.load(std::memory_order_acquire);
            for (uint64_t i = answered; i < n_sub; ++i)
                if (egtb_serve_wait(S, tickets[i], 60000, nullptr) != EGTB_OK) break;
            throw Error(EGTB_ERR_TIMEOUT, "replay: request " + std::to_string(answered) + " not answered" +
                                              " (ranges still used by unanswered requests stay registered)");
        }
        driver.join();
        if (failed) throw Error(EGTB_ERR_ARG, "replay: a request was rejected");
        if (wall_us) *wall_us = std::chrono::duration<double, std::micro>(Clock::now() - t0).count();
    });
}

extern "C" int egtb_serve_stop(egtb_server *S) {
    return guarded([&] {
        if (!S) return;
        S->stop = true;
        if (S->worker.joinable()) S->worker.join();
        cudaSetDevice(S->device);
        for (auto &sl : S->slots) {
            if (sl.stream) cudaStreamSynchronize(sl.stream);
            cudaFreeHost(sl.h_pos);
            cudaFreeHost(sl.h_out);
            cudaFreeHost(sl.h_valid);
            cudaFree(sl.d_pos);
            cudaFree(sl.d_out);
            cudaFree(sl.d_valid);
            cudaFreeHost(sl.h_reqs);
            cudaFree(sl.d_reqs);
            if (sl.event) cudaEventDestroy(sl.event);
            if (sl.stream) cudaStreamDestroy(sl.stream);
        }
        for (auto &r : S->registered) cudaHostUnregister((void *)r.begin);
        delete S;
    });
}
