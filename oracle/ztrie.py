"""CPU restatement of the reference's compressed book format and its search.

TEST INFRASTRUCTURE ONLY (the checker of the library's compressed books; the
product never imports it).

Restates, from the reference project:
  * build_trie_index (native_core/src/TrieCompression.cpp:115-191): a byte
    trie over bytes 7, 6, 5, 4 of the sorted boards; every level starts with
    an empty entry, every entry holds its byte and the index of its last
    child (byte-4 level: of its last book entry);
  * compress_and_save_serial / get_segment_positions (:193-275): blocks cut
    after the byte-4 group that takes a block past 32768 entries, byte-4
    `next` made relative to the block (0 for a block's last group), each
    block's {u32 low; T rate} entries xz-compressed (NativeLzma.cpp:141-161:
    lzma_easy_buffer_encode, preset 1, CRC64 check);
  * trie_compress_typed (:312-354): the i / ii / s / z files;
  * maybe_do_compress_classic (native_core/src/CompressionBridge.cpp:41-59):
    which books are compressed;
  * trie_search_with_context (native_core/src/ReaderRuntime.cpp:318-477):
    the reader's search, with its range rules as they are.

xz coding goes through liblzma (xz-utils' liblzma.so.5, the library the
reference loads at run time), called through ctypes with the reference's
arguments. Pinned by tests/test_oracle_golden.py against the digests of the
reference's own compressed builds (tests/golden/cases.json).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

BLOCK_ENTRIES = 32768
MIN_BYTES = 2097152
RATE = {"uint32": "<u4", "uint64": "<u8", "float32": "<f4", "float64": "<f8", "1-float32": "<f4",
        "1-float64": "<f8"}

_xz = None


def _lib():
    global _xz
    if _xz is None:
        L = ctypes.CDLL("liblzma.so.5")
        L.lzma_stream_buffer_bound.restype = ctypes.c_size_t
        L.lzma_stream_buffer_bound.argtypes = [ctypes.c_size_t]
        L.lzma_easy_buffer_encode.restype = ctypes.c_int
        L.lzma_easy_buffer_encode.argtypes = [ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p, ctypes.c_char_p,
                                              ctypes.c_size_t, ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t),
                                              ctypes.c_size_t]
        L.lzma_version_string.restype = ctypes.c_char_p
        _xz = L
    return _xz


def liblzma_version() -> str:
    return _lib().lzma_version_string().decode()


def xz_encode(data: bytes) -> bytes:
    L = _lib()
    cap = L.lzma_stream_buffer_bound(len(data))
    out = ctypes.create_string_buffer(cap)
    pos = ctypes.c_size_t(0)
    rc = L.lzma_easy_buffer_encode(1, 4, None, data, len(data), out, ctypes.byref(pos), cap)  # preset 1, CRC64
    if rc != 0:
        raise RuntimeError(f"lzma_easy_buffer_encode failed ({rc})")
    return out.raw[:pos.value]


def xz_decode(data: bytes) -> bytes:
    import lzma
    return lzma.decompress(data, format=lzma.FORMAT_XZ)


def wants_compression(book_name: str, nbytes: int) -> bool:
    if not book_name.endswith("book"):
        return False
    if book_name.endswith(("_0.book", "_1.book", "_2.book")):
        return False
    return nbytes > MIN_BYTES


def compress_book(book: bytes, dtype: str, stem: str) -> dict:
    """The four files of a book's .z directory, {name: bytes}; stem is the
    book's file name without "book" (e.g. "442_512_100.")."""
    rt = np.dtype(RATE[dtype])
    rec = np.dtype([("key", "<u8"), ("rate", rt)])
    rows = np.frombuffer(book, dtype=rec)
    keys = rows["key"]
    n = len(keys)
    lv = [[(0, 0)] for _ in range(4)]
    byte = [((keys >> np.uint64(56 - 8 * m)) & np.uint64(0xFF)).astype(np.uint8) for m in range(4)]
    # first level (0..3) whose byte changes between entry j-1 and j; 4 = none
    change = np.full(n, 4, dtype=np.int64)
    for m in range(3, -1, -1):
        diff = np.zeros(n, dtype=bool)
        diff[1:] = byte[m][1:] != byte[m][:-1]
        change[diff] = m

    def close(frm, last):
        for m in range(frm, 4):
            lv[m].append((int(byte[m][last]), len(lv[m + 1]) if m < 3 else last))

    for j in np.nonzero(change[1:] < 4)[0] + 1:
        close(int(change[j]), int(j) - 1)
    close(0, n - 1)
    g3 = [list(e) for e in lv[3]]
    blocks, ends, start = [], [], 0
    for i in range(1, len(g3) - 1):
        end = g3[i][1] + 1
        if end - start > BLOCK_ENTRIES:
            blocks.append((start, end))
            ends.append(i)
            g3[i][1] = 0
            start = end
        else:
            g3[i][1] -= start
    g3[-1][1] = 0
    blocks.append((start, n))
    ends.append(len(g3) - 1)
    crec = np.dtype([("low", "<u4"), ("rate", rt)])
    z, seg, at = [], [(0, 0)], 0
    for (lo, hi), e in zip(blocks, ends):
        c = np.zeros(hi - lo, dtype=crec)
        c["low"] = (keys[lo:hi] & np.uint64(0xFFFFFFFF)).astype(np.uint32)
        c["rate"] = rows["rate"][lo:hi]
        blob = xz_encode(c.tobytes())
        z.append(blob)
        at += len(blob)
        seg.append((e, at))
    node32 = np.dtype([("key", "u1"), ("next", "<u4")])
    node16 = np.dtype([("key", "u1"), ("next", "<u2")])
    segd = np.dtype([("index", "<u4"), ("offset", "<u8")])
    base1 = 1 + len(lv[0])
    base2 = base1 + len(lv[1])
    ind = [(0, 1)] + [(k, nx + base1) for k, nx in lv[0]] + [(k, nx + base2) for k, nx in lv[1]] + list(lv[2])
    return {
        stem + "i": np.array(ind, dtype=node32).tobytes(),
        stem + "ii": np.array([(k, nx & 0xFFFF) for k, nx in g3], dtype=node16).tobytes(),
        stem + "s": np.array(seg, dtype=segd).tobytes(),
        stem + "z": b"".join(z),
    }


class TrieLayer:
    """A .z directory read back for searching."""

    def __init__(self, files: dict, stem: str, dtype: str):
        node32 = np.dtype([("key", "u1"), ("next", "<u4")])
        node16 = np.dtype([("key", "u1"), ("next", "<u2")])
        segd = np.dtype([("index", "<u4"), ("offset", "<u8")])
        self.ind = np.frombuffer(files[stem + "i"], dtype=node32)
        self.ii = np.frombuffer(files[stem + "ii"], dtype=node16)
        self.seg = np.frombuffer(files[stem + "s"], dtype=segd)
        self.z = files[stem + "z"]
        self.crec = np.dtype([("low", "<u4"), ("rate", RATE[dtype])])
        self._blocks = {}

    @classmethod
    def from_dir(cls, zdir: str, stem: str, dtype: str) -> "TrieLayer":
        files = {stem + s: open(os.path.join(zdir, stem + s), "rb").read() for s in ("i", "ii", "s", "z")}
        return cls(files, stem, dtype)

    def _block(self, start: int, end: int):
        if (start, end) not in self._blocks:
            self._blocks[(start, end)] = np.frombuffer(xz_decode(self.z[start:end]), dtype=self.crec) \
                if end > start else np.zeros(0, dtype=self.crec)
        return self._blocks[(start, end)]

    def search(self, board: int):
        """trie_search_with_context: the stored rate, or None for a miss
        (the caller reads a miss as the dtype's zero)."""
        ind, ii, seg = self.ind, self.ii, self.seg
        if len(ind) < 2 or len(seg) < 2:
            return None
        low, high = 2, int(ind[1]["next"]) - 1
        for m in range(3):
            want = (board >> (56 - 8 * m)) & 0xFF
            found, mid = False, low
            while low <= high:
                mid = (low + high) // 2
                k = int(ind[mid]["key"])
                if k == want:
                    found = True
                    break
                if k < want:
                    low = mid + 1
                else:
                    if mid == 0:
                        break
                    high = mid - 1
            if not found:
                return None
            low, high = int(ind[mid - 1]["next"]) + 1, int(ind[mid]["next"])
        part = ii[low - 1:high + 1]
        want4 = (board >> 32) & 0xFF
        if len(part) <= 1:
            return None
        lo, hi, pos = 1, len(part) - 1, None
        while lo <= hi:
            mid = (lo + hi) // 2
            k = int(part[mid]["key"])
            if k == want4:
                pos = mid - 1
                break
            if k < want4:
                lo = mid + 1
            else:
                if mid == 0:
                    break
                hi = mid - 1
        if pos is None:
            return None
        target = pos + low
        a, c, start, end = 0, len(seg) - 1, 0, 0
        while a <= c:
            mid = (a + c) // 2
            if int(seg[mid]["index"]) < target:
                a = mid + 1
            else:
                start, end = int(seg[mid - 1]["offset"]), int(seg[mid]["offset"])
                if mid == 0:
                    break
                c = mid - 1
        block = self._block(start, end)
        t32 = board & 0xFFFFFFFF
        sub_low = int(part[pos]["next"])
        sub_high = int(part[pos + 1]["next"]) + 1
        if sub_high == 1:
            if len(block) and t32 == int(block[0]["low"]):
                return block[0]["rate"].item()
            sub_high = len(block)
        if sub_low != 0:
            sub_low += 1
        while sub_low < sub_high:
            mid = (sub_low + sub_high) // 2
            if int(block[mid]["low"]) < t32:
                sub_low = mid + 1
            else:
                sub_high = mid
        if sub_low < len(block) and int(block[sub_low]["low"]) == t32:
            return block[sub_low]["rate"].item()
        return None
