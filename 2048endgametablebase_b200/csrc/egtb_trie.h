// Compressed books: the reference's on-disk format for large layers, a byte
// trie over the top four bytes of the boards plus xz blocks of the remaining
// {low 32 bits, rate} entries (TrieCompression.cpp:115-354 writes it,
// ReaderRuntime.cpp:318-477 reads it). A layer <name>_<t>.book becomes the
// directory <name>_<t>.z holding <name>_<t>.{i,ii,s,z}:
//   i   packed {u8 key; u32 next}: a root entry, then the levels of bytes 7,
//       6 and 5, each entry's `next` the index (in this file) of its last
//       child; byte-5 entries point into ii
//   ii  packed {u8 key; u16 next}: byte-4 groups, `next` the group's last
//       entry relative to its xz block (0 for a block's last group)
//   s   packed {u32 index; u64 offset}: per xz block, the ii entry that ends
//       it and the end of its bytes in z
//   z   the xz streams (preset 1, CRC64 check) of the blocks' packed
//       {u32 low; T rate} entries, one after another
// liblzma is loaded at run time (liblzma.so.5), as the reference does.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace egtb {

// liblzma present and usable (why: the reason when not).
bool xz_available(std::string *why = nullptr);

// The rule of maybe_do_compress_classic (CompressionBridge.cpp:41-59): a
// .book file other than layers 0, 1, 2, larger than 2 MiB.
bool book_wants_compression(const std::string &book_path, unsigned long long bytes);

// Write the .z directory of one book from its packed records (rec = 8 +
// rate_bytes bytes each, ascending boards), with `threads` threads
// compressing blocks. An existing directory of that name is replaced.
void write_compressed_book(const std::string &book_path, const unsigned char *records, size_t n,
                           size_t rate_bytes, int threads);

// Compress every layer file of a finished table that the rule selects and
// remove its .book (the compression pass of the solve, BookSolver.cpp:596-597,
// and of the optimal-branch pass, :720-728, applied once the books are final).
void compress_table_books(const std::string &pathname, int steps, size_t rate_bytes, int threads);

// A compressed layer read back: the trie levels, the block table and every
// block decoded, entries in file order.
struct TrieLayer {
    std::vector<uint8_t> i_key;
    std::vector<uint32_t> i_next;
    std::vector<uint8_t> ii_key;
    std::vector<uint16_t> ii_next;
    std::vector<uint32_t> seg_index;     // s entries' ii index
    std::vector<uint64_t> block_end;     // entries decoded up to and including block k (k = s entry)
    std::vector<uint32_t> low;           // decoded entries: low 32 bits of the board
    std::vector<unsigned char> rates;    // ... and their rates (rate_bytes each)
};

// Read <dir>/<stem>{i,ii,s,z} (stem = the .book file name without "book").
// False when a file is missing or a block does not decode.
bool read_compressed_book(const std::string &zdir, const std::string &stem, size_t rate_bytes, TrieLayer &out,
                          int threads);

}  // namespace egtb
