"""Parquet data pages decoded on the GPU into Arrow columns: the scan side
that feeds `GpuHashAggregate` without a trip through host memory.

Mirrors the reference's page decoder (ParquetPageDecoder.decode,
parquet/src/main/java/io/vecruntime/parquet/codec/ParquetPageDecoder.java:214-266;
RleBitPackingReader.java) for flat columns, through libvrgpu's vr_pq_*:
a dictionary-encoded page decodes to its ids, which go to the aggregate as a
VR_DICT32 column with the column chunk's dictionary attached
(`dictionary_page` decodes a BYTE_ARRAY dictionary page into one); a PLAIN
page of a fixed-width type decodes to its values. A null slot holds 0.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import native as N
from .columns import Dictionary

PLAIN = N.VR_PQ_PLAIN
RLE_DICTIONARY = N.VR_PQ_RLE_DICTIONARY


@dataclass
class Page:
    """One decompressed data page in device memory (`data`: a device
    pointer). v1: [int32 byte length of the levels][levels][values]; v2:
    [levels (levels_length bytes)][values]; no levels when max_def_level is 0."""
    data: int
    length: int
    num_values: int
    max_def_level: int = 0
    v2: bool = False
    levels_length: int = 0
    encoding: int = RLE_DICTIONARY
    value_bytes: int = 4

    def ctypes(self) -> N.PqPage:
        return N.PqPage(self.data, self.length, self.num_values, self.max_def_level, 1 if self.v2 else 0,
                        self.levels_length, self.encoding, self.value_bytes)


class PageDecoder:
    """A device page decoder sized for calls of up to `max_values` slots and
    `max_bytes` page bytes (vr_pq_create)."""

    def __init__(self, max_values: int, max_bytes: int, device: int = 0):
        self._lib = N.lib()
        h = C.c_void_p()
        N.check(self._lib.vr_pq_create(device, max_values, max_bytes, C.byref(h)), "vr_pq_create")
        self.h = h
        self.device = device

    @staticmethod
    def descriptors(pages: Sequence[Page]):
        """The pages as the vr_pq_page array the library reads: build it once
        for a chunk decoded more than once (thousands of pages cost the
        Python loop more than the decode)."""
        return (N.PqPage * max(1, len(pages)))(*[p.ctypes() for p in pages])

    def decode(self, pages, out_data: int, out_validity: Optional[int], stream: int = 0) -> None:
        """Decodes `pages` (one column chunk, in order: Page objects or the
        array `descriptors` returns) into the device buffers `out_data`
        (value_bytes per slot) and `out_validity` (LSB-first bitmap);
        asynchronous on `stream`."""
        arr = pages if isinstance(pages, C.Array) else self.descriptors(pages)
        N.check(self._lib.vr_pq_decode(self.h, len(pages), arr, C.c_void_p(out_data),
                                       C.c_void_p(out_validity) if out_validity else None,
                                       C.c_void_p(stream) if stream else None), "vr_pq_decode")

    def sync(self) -> int:
        """Waits for the last decode; returns its present (non-null) slots.
        A malformed page raises with the page and the reason."""
        n = C.c_int64()
        N.check(self._lib.vr_pq_sync(self.h, C.byref(n)), "vr_pq_sync")
        return n.value

    def decode_to_tensors(self, pages: Sequence[Page], stream: int = 0):
        """Decodes into fresh device tensors: (data, validity or None,
        present slots). `data` is int32 for dictionary pages."""
        import torch

        n = sum(p.num_values for p in pages)
        vb = 4 if pages and pages[0].encoding == RLE_DICTIONARY else (pages[0].value_bytes if pages else 4)
        dev = torch.device("cuda", self.device)
        data = torch.empty(max(n, 1) * vb + 16, dtype=torch.uint8, device=dev)
        levels = any(p.max_def_level > 0 for p in pages)
        # whole 4-byte words of the bitmap stay inside the buffer
        valid = torch.zeros(((n + 7) // 8 + 15) // 16 * 16 + 16, dtype=torch.uint8, device=dev) if levels else None
        self.decode(pages, data.data_ptr(), valid.data_ptr() if valid is not None else None, stream)
        present = self.sync()
        return data, valid, present

    def close(self) -> None:
        if self.h:
            self._lib.vr_pq_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def dictionary_page(page: bytes, num_values: int) -> Dictionary:
    """A PLAIN BYTE_ARRAY dictionary page (host bytes) as the Dictionary a
    VR_DICT32 column carries (vr_pq_plain_dictionary;
    ParquetPageDecoder.decodeDictionary, ParquetPageDecoder.java:440-513)."""
    lib = N.lib()
    buf = C.create_string_buffer(bytes(page), max(1, len(page)))
    total = C.c_int64()
    N.check(lib.vr_pq_plain_dictionary(buf, len(page), num_values, None, None, C.byref(total)),
            "vr_pq_plain_dictionary")
    offsets = np.zeros(num_values + 1, np.int32)
    data = np.zeros(total.value + 16, np.uint8)
    N.check(lib.vr_pq_plain_dictionary(buf, len(page), num_values, offsets.ctypes.data, data.ctypes.data,
                                       C.byref(total)), "vr_pq_plain_dictionary")
    return Dictionary(offsets, data)
