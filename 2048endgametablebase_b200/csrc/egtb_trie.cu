// Compressed books (see egtb_trie.h): host side. The trie is built in one
// pass over the sorted boards; blocks are cut at byte-4 group ends once they
// pass 32768 entries and xz-compressed by a pool of threads; reading decodes
// every block of a layer for the device-resident reader.
#include "egtb_trie.h"

#include <dlfcn.h>
#include <sys/stat.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <limits>
#include <mutex>
#include <thread>

#include "egtb_host.h"

namespace fs = std::filesystem;

namespace egtb {

// ------------------------------------------------------------- liblzma ----
//
// Three entry points of liblzma's stable C API, resolved by name: the
// single-call xz encoder and decoder and the output bound. Enum arguments
// are passed as their integer values (preset 1; check CRC64 = 4; return
// 0 = OK, 10 = output buffer too small).

namespace {

struct XzApi {
    void *so = nullptr;
    size_t (*bound)(size_t) = nullptr;
    int (*encode)(uint32_t, int, const void *, const uint8_t *, size_t, uint8_t *, size_t *, size_t) = nullptr;
    int (*decode)(uint64_t *, uint32_t, const void *, const uint8_t *, size_t *, size_t, uint8_t *, size_t *,
                  size_t) = nullptr;
    std::string why;
};

constexpr uint32_t kXzPreset = 1;
constexpr int kXzCheckCrc64 = 4;
constexpr int kXzOk = 0;
constexpr int kXzBufError = 10;
constexpr size_t kBlockEntries = 32768;           // a block closes once it passes this many entries
constexpr unsigned long long kMinBytes = 2097152;  // books up to 2 MiB stay .book

const XzApi &xz() {
    static XzApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        for (const char *name : {"liblzma.so.5", "liblzma.so"}) {
            api.so = dlopen(name, RTLD_NOW | RTLD_LOCAL);
            if (api.so) break;
        }
        if (!api.so) {
            api.why = "liblzma.so.5 not found";
            return;
        }
        api.bound = reinterpret_cast<size_t (*)(size_t)>(dlsym(api.so, "lzma_stream_buffer_bound"));
        api.encode = reinterpret_cast<decltype(api.encode)>(dlsym(api.so, "lzma_easy_buffer_encode"));
        api.decode = reinterpret_cast<decltype(api.decode)>(dlsym(api.so, "lzma_stream_buffer_decode"));
        if (!api.bound || !api.encode || !api.decode) api.why = "liblzma lacks the single-call xz API";
    });
    return api;
}

std::vector<uint8_t> xz_encode(const uint8_t *data, size_t n) {
    const XzApi &a = xz();
    if (!a.why.empty()) throw Error(EGTB_ERR_UNSUPPORTED, "compressed books need liblzma: " + a.why);
    std::vector<uint8_t> out(a.bound(n));
    size_t pos = 0;
    const int rc = a.encode(kXzPreset, kXzCheckCrc64, nullptr, data, n, out.data(), &pos, out.size());
    if (rc != kXzOk) throw Error(EGTB_ERR_IO, "xz encode failed (" + std::to_string(rc) + ")");
    out.resize(pos);
    return out;
}

bool xz_decode(const uint8_t *data, size_t n, std::vector<uint8_t> &out) {
    const XzApi &a = xz();
    if (!a.why.empty()) throw Error(EGTB_ERR_UNSUPPORTED, "compressed books need liblzma: " + a.why);
    size_t cap = std::max<size_t>(n * 8, 4096);
    for (int attempt = 0; attempt < 12; ++attempt) {
        out.resize(cap);
        uint64_t memlimit = std::numeric_limits<uint64_t>::max();
        size_t in_pos = 0, out_pos = 0;
        const int rc = a.decode(&memlimit, 0, nullptr, data, &in_pos, n, out.data(), &out_pos, out.size());
        if (rc == kXzOk) {
            out.resize(out_pos);
            return true;
        }
        if (rc != kXzBufError) return false;
        cap *= 2;
    }
    return false;
}

#pragma pack(push, 1)
struct INode {
    uint8_t key;
    uint32_t next;
};
struct IINode {
    uint8_t key;
    uint16_t next;
};
struct SegEntry {
    uint32_t index;
    uint64_t offset;
};
#pragma pack(pop)
static_assert(sizeof(INode) == 5 && sizeof(IINode) == 3 && sizeof(SegEntry) == 12, "packed trie records");

struct Group {
    uint8_t key;
    uint64_t next;
};

void put_file(const std::string &path, const void *data, size_t bytes) {
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f) throw Error(EGTB_ERR_IO, "cannot open " + path);
    if (bytes) f.write(static_cast<const char *>(data), (std::streamsize)bytes);
    if (!f) throw Error(EGTB_ERR_IO, "write failed: " + path);
}

bool get_file(const std::string &path, std::vector<unsigned char> &out) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) return false;
    const std::streamsize n = f.tellg();
    f.seekg(0);
    out.resize((size_t)n);
    if (n && !f.read(reinterpret_cast<char *>(out.data()), n)) return false;
    return true;
}

// Run job(k) for k in [0, n) on up to `threads` threads.
template <typename F>
void parallel_for(size_t n, int threads, F &&job) {
    const int t = (int)std::max<size_t>(1, std::min<size_t>(n, (size_t)std::max(1, threads)));
    std::atomic<size_t> next{0};
    std::mutex err_mu;
    std::exception_ptr err;
    auto worker = [&] {
        for (size_t k; (k = next.fetch_add(1)) < n;) {
            try {
                job(k);
            } catch (...) {
                std::lock_guard<std::mutex> lk(err_mu);
                if (!err) err = std::current_exception();
            }
        }
    };
    std::vector<std::thread> pool;
    for (int i = 1; i < t; ++i) pool.emplace_back(worker);
    worker();
    for (auto &th : pool) th.join();
    if (err) std::rethrow_exception(err);
}

std::string zdir_of(const std::string &book_path) {
    fs::path p(book_path);
    p.replace_extension(".z");
    return p.string();
}

std::string stem_of(const std::string &book_path) {
    const std::string f = fs::path(book_path).filename().string();
    return f.substr(0, f.size() - 4);  // "<name>_<t>.book" -> "<name>_<t>."
}

bool ends_with(const std::string &s, const char *suffix) {
    const size_t n = std::strlen(suffix);
    return s.size() >= n && s.compare(s.size() - n, n, suffix) == 0;
}

}  // namespace

bool xz_available(std::string *why) {
    const XzApi &a = xz();
    if (why) *why = a.why;
    return a.why.empty();
}

bool book_wants_compression(const std::string &book_path, unsigned long long bytes) {
    if (!ends_with(book_path, "book")) return false;
    if (ends_with(book_path, "_0.book") || ends_with(book_path, "_1.book") || ends_with(book_path, "_2.book"))
        return false;
    return bytes > kMinBytes;
}

void write_compressed_book(const std::string &book_path, const unsigned char *records, size_t n, size_t rate_bytes,
                           int threads) {
    if (n == 0) return;
    const size_t rec = 8 + rate_bytes;
    auto board = [&](size_t j) {
        uint64_t k;
        std::memcpy(&k, records + j * rec, 8);
        return k;
    };
    auto byte_of = [](uint64_t k, int level) { return (uint8_t)(k >> (56 - 8 * level)); };
    // levels 0..3 = bytes 7..4; every level starts with an empty root entry
    std::vector<Group> lv[4];
    for (auto &v : lv) v.push_back({0, 0});
    // groups of levels `from`..3 end at entry `last`: each gets its byte and
    // the index of its last child one level down (level 3: its last entry)
    auto close = [&](int from, size_t last) {
        const uint64_t k = board(last);
        for (int m = from; m < 4; ++m)
            lv[m].push_back({byte_of(k, m), m < 3 ? (uint64_t)lv[m + 1].size() : (uint64_t)last});
    };
    uint64_t prev = board(0);
    for (size_t j = 1; j < n; ++j) {
        const uint64_t k = board(j);
        int m = 0;
        while (m < 4 && byte_of(k, m) == byte_of(prev, m)) ++m;
        if (m < 4) close(m, j - 1);
        prev = k;
    }
    close(0, n - 1);
    // blocks: cut after the byte-4 group that takes a block past kBlockEntries;
    // a group's `next` becomes relative to its block (0 for a block's last)
    std::vector<Group> &g3 = lv[3];
    std::vector<std::pair<size_t, size_t>> blocks;
    std::vector<uint32_t> ends;
    size_t start = 0;
    for (size_t i = 1; i + 1 < g3.size(); ++i) {
        const size_t end = (size_t)g3[i].next + 1;
        if (end - start > kBlockEntries) {
            blocks.push_back({start, end});
            ends.push_back((uint32_t)i);
            g3[i].next = 0;
            start = end;
        } else {
            g3[i].next -= start;
        }
    }
    g3.back().next = 0;
    blocks.push_back({start, n});
    ends.push_back((uint32_t)(g3.size() - 1));
    // block payloads {u32 low; rate}, compressed in parallel
    std::vector<std::vector<uint8_t>> z(blocks.size());
    const size_t crec = 4 + rate_bytes;
    parallel_for(blocks.size(), threads, [&](size_t b) {
        const size_t lo = blocks[b].first, hi = blocks[b].second;
        std::vector<uint8_t> buf((hi - lo) * crec);
        for (size_t j = lo; j < hi; ++j) {
            const uint32_t low = (uint32_t)board(j);
            std::memcpy(buf.data() + (j - lo) * crec, &low, 4);
            std::memcpy(buf.data() + (j - lo) * crec + 4, records + j * rec + 8, rate_bytes);
        }
        z[b] = xz_encode(buf.data(), buf.size());
    });
    // files
    const std::string dir = zdir_of(book_path), prefix = dir + "/" + stem_of(book_path);
    std::error_code ec;
    fs::remove_all(dir, ec);
    fs::create_directories(dir, ec);
    if (ec) throw Error(EGTB_ERR_IO, "cannot create " + dir + ": " + ec.message());
    std::vector<SegEntry> seg{{0u, 0ull}};
    {
        std::ofstream f(prefix + "z", std::ios::binary | std::ios::trunc);
        if (!f) throw Error(EGTB_ERR_IO, "cannot open " + prefix + "z");
        uint64_t at = 0;
        for (size_t b = 0; b < z.size(); ++b) {
            f.write(reinterpret_cast<const char *>(z[b].data()), (std::streamsize)z[b].size());
            at += z[b].size();
            seg.push_back({ends[b], at});
        }
        if (!f) throw Error(EGTB_ERR_IO, "write failed: " + prefix + "z");
    }
    std::vector<IINode> ii(g3.size());
    for (size_t i = 0; i < g3.size(); ++i) ii[i] = {g3[i].key, (uint16_t)g3[i].next};
    // i: a root entry, then levels 0, 1, 2 with `next` turned into indexes of
    // this file (level 2 keeps its indexes into ii)
    std::vector<INode> in;
    in.reserve(1 + lv[0].size() + lv[1].size() + lv[2].size());
    in.push_back({0, 1u});
    const uint32_t base1 = 1u + (uint32_t)lv[0].size(), base2 = base1 + (uint32_t)lv[1].size();
    for (const Group &e : lv[0]) in.push_back({e.key, (uint32_t)e.next + base1});
    for (const Group &e : lv[1]) in.push_back({e.key, (uint32_t)e.next + base2});
    for (const Group &e : lv[2]) in.push_back({e.key, (uint32_t)e.next});
    put_file(prefix + "ii", ii.data(), ii.size() * sizeof(IINode));
    put_file(prefix + "i", in.data(), in.size() * sizeof(INode));
    put_file(prefix + "s", seg.data(), seg.size() * sizeof(SegEntry));
}

void compress_table_books(const std::string &pathname, int steps, size_t rate_bytes, int threads) {
    const size_t rec = 8 + rate_bytes;
    for (int t = 0; t < steps; ++t) {
        const std::string path = pathname + std::to_string(t) + ".book";
        struct stat st;
        if (::stat(path.c_str(), &st) != 0 || !S_ISREG(st.st_mode)) continue;
        if (!book_wants_compression(path, (unsigned long long)st.st_size)) continue;
        std::vector<unsigned char> data;
        if (!get_file(path, data)) throw Error(EGTB_ERR_IO, "cannot read " + path);
        if (data.size() % rec) continue;
        write_compressed_book(path, data.data(), data.size() / rec, rate_bytes, threads);
        std::error_code ec;
        fs::remove(path, ec);
    }
}

bool read_compressed_book(const std::string &zdir, const std::string &stem, size_t rate_bytes, TrieLayer &out,
                          int threads) {
    const std::string prefix = zdir + "/" + stem;
    std::vector<unsigned char> fi, fii, fs_, fz;
    if (!get_file(prefix + "i", fi) || !get_file(prefix + "ii", fii) || !get_file(prefix + "s", fs_) ||
        !get_file(prefix + "z", fz))
        return false;
    const size_t ni = fi.size() / sizeof(INode), nii = fii.size() / sizeof(IINode), ns = fs_.size() / sizeof(SegEntry);
    out.i_key.resize(ni);
    out.i_next.resize(ni);
    for (size_t k = 0; k < ni; ++k) {
        INode e;
        std::memcpy(&e, fi.data() + k * sizeof e, sizeof e);
        out.i_key[k] = e.key;
        out.i_next[k] = e.next;
    }
    out.ii_key.resize(nii);
    out.ii_next.resize(nii);
    for (size_t k = 0; k < nii; ++k) {
        IINode e;
        std::memcpy(&e, fii.data() + k * sizeof e, sizeof e);
        out.ii_key[k] = e.key;
        out.ii_next[k] = e.next;
    }
    std::vector<SegEntry> seg(ns);
    if (ns) std::memcpy(seg.data(), fs_.data(), ns * sizeof(SegEntry));
    out.seg_index.resize(ns);
    for (size_t k = 0; k < ns; ++k) out.seg_index[k] = seg[k].index;
    // block k (k >= 1) is z[seg[k-1].offset, seg[k].offset)
    const size_t crec = 4 + rate_bytes;
    std::vector<std::vector<uint8_t>> dec(ns);
    std::atomic<bool> bad{false};
    parallel_for(ns > 0 ? ns - 1 : 0, threads, [&](size_t b) {
        const uint64_t lo = seg[b].offset, hi = seg[b + 1].offset;
        if (hi < lo || hi > fz.size() || !xz_decode(fz.data() + lo, hi - lo, dec[b + 1]) || dec[b + 1].size() % crec)
            bad = true;
    });
    if (bad) return false;
    out.block_end.assign(ns, 0);
    size_t total = 0;
    for (size_t k = 1; k < ns; ++k) {
        total += dec[k].size() / crec;
        out.block_end[k] = total;
    }
    out.low.resize(total);
    out.rates.resize(total * rate_bytes);
    size_t at = 0;
    for (size_t k = 1; k < ns; ++k)
        for (size_t j = 0; j < dec[k].size() / crec; ++j, ++at) {
            std::memcpy(&out.low[at], dec[k].data() + j * crec, 4);
            std::memcpy(out.rates.data() + at * rate_bytes, dec[k].data() + j * crec + 4, rate_bytes);
        }
    return true;
}

}  // namespace egtb
