// Link-time stand-in for the reference's NativeLzma.cpp when building the
// reference's formation_core module as a CPU oracle.
//
// The reference's NativeLzma.cpp (native_core/src/NativeLzma.cpp) needs
// liblzma headers, which this image does not have. Compression is off by
// default in the reference (RunOptions::compress = false,
// native_core/include/FormationRuntime.h:29) and is not on the classic
// build/lookup path, so these definitions only satisfy the linker: every
// call reports failure, exactly as the reference does when xz is absent.
//
// Declarations: native_core/include/NativeLzma.h.

#include <cstddef>
#include <cstdint>
#include <optional>
#include <stdexcept>
#include <string>
#include <vector>

bool compress_with_7z_or_xz(const std::string &, int) { return false; }

bool decompress_with_7z_or_xz(const std::string &) { return false; }

std::vector<uint8_t> compress_xz_block_native(const uint8_t *, size_t, int) {
    throw std::runtime_error("xz compression is not built into this oracle");
}

std::vector<uint8_t> decompress_xz_block_native(const uint8_t *, size_t) {
    throw std::runtime_error("xz decompression is not built into this oracle");
}

bool compress_uint64_array_native(const std::vector<uint64_t> &, const std::string &, int) { return false; }

std::vector<uint64_t> decompress_uint64_array_native(const std::string &) {
    throw std::runtime_error("xz decompression is not built into this oracle");
}

std::optional<size_t> find_value_uint64_compressed_native(const std::string &, uint64_t) { return std::nullopt; }
