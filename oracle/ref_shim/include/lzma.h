/*
 * Type-only stand-in for xz's <lzma.h>, for compiling the reference's
 * NativeLzma.cpp (native_core/src/NativeLzma.cpp) into the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY. The reference loads liblzma.so.5 at run time
 * with dlopen/dlsym (NativeLzma.cpp:88-131) and uses the header only for
 * these types and constants, so this file declares no functions. The
 * names and values are those of liblzma's public API (lzma/base.h,
 * lzma/check.h of xz 5.x), which are fixed by its ABI.
 */
#ifndef EGTB_ORACLE_LZMA_SHIM_H
#define EGTB_ORACLE_LZMA_SHIM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    LZMA_OK = 0,
    LZMA_STREAM_END = 1,
    LZMA_NO_CHECK = 2,
    LZMA_UNSUPPORTED_CHECK = 3,
    LZMA_GET_CHECK = 4,
    LZMA_MEM_ERROR = 5,
    LZMA_MEMLIMIT_ERROR = 6,
    LZMA_FORMAT_ERROR = 7,
    LZMA_OPTIONS_ERROR = 8,
    LZMA_DATA_ERROR = 9,
    LZMA_BUF_ERROR = 10,
    LZMA_PROG_ERROR = 11
} lzma_ret;

typedef enum {
    LZMA_CHECK_NONE = 0,
    LZMA_CHECK_CRC32 = 1,
    LZMA_CHECK_CRC64 = 4,
    LZMA_CHECK_SHA256 = 10
} lzma_check;

typedef struct {
    void *(*alloc)(void *opaque, size_t nmemb, size_t size);
    void (*free)(void *opaque, void *ptr);
    void *opaque;
} lzma_allocator;

#ifdef __cplusplus
}
#endif
#endif
