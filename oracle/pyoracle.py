"""ctypes binding of the CPU oracle (oracle/_build/liborc.so).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use it as the checker / the timed CPU port; the product
path never does. Shares only the ABI structs (include/vrgpu.h) with it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from vecruntime_b200 import native as N

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liborc.so")

ORC_FP_SEQUENTIAL = 0
ORC_FP_COMPENSATED = 1

_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.orc_agg_create.argtypes = [C.POINTER(N.AggSpec), C.POINTER(P)]
        L.orc_agg_update.argtypes = [P, C.POINTER(N.Batch), C.c_int64]
        L.orc_agg_num_groups.argtypes = [P]
        L.orc_agg_num_groups.restype = C.c_int64
        L.orc_agg_num_outputs.argtypes = [P]
        L.orc_agg_output_type.argtypes = [P, C.c_int, C.POINTER(N.ColumnType)]
        L.orc_agg_emit.argtypes = [P, C.c_int64, C.c_int64, C.POINTER(N.OutColumn), C.c_int]
        L.orc_agg_merge.argtypes = [P, P]
        L.orc_agg_destroy.argtypes = [P]
        L.orc_agg_destroy.restype = None
        L.orc_last_error.restype = C.c_char_p
        L.orc_hash_rows.argtypes = [C.c_int32, C.POINTER(N.ColumnType), C.POINTER(N.Column), C.c_int64, P, C.c_int32]
        L.orc_agg_key_dictionary.argtypes = [P, C.c_int32, C.POINTER(C.c_int32), P, P, C.c_int64,
                                              C.POINTER(C.c_int64)]
        L.orc_agg_update_threads.argtypes = [P, C.POINTER(N.Batch), C.c_int32, C.c_int64]
        L.orc_agg_run_threads.argtypes = [C.POINTER(N.AggSpec), C.POINTER(N.Batch), C.c_int32, C.c_int64,
                                          C.POINTER(C.c_double), C.POINTER(C.c_int64)]
        L.orc_rle_decode.argtypes = [P, C.c_int64, C.c_int32, C.c_int64, P]
        L.orc_pq_decode_page.argtypes = [P, C.POINTER(N.PqPage), P, P, C.POINTER(C.c_int64)]
        L.orc_pq_plain_dictionary.argtypes = [P, C.c_int64, C.c_int32, P, P, C.POINTER(C.c_int64)]
        L.orc_pq_last_error.restype = C.c_char_p
        L.orc_pq_decode_pages_threads.argtypes = [C.c_int32, P, C.POINTER(N.PqPage), P, P, P, P, C.c_int32,
                                                  C.POINTER(C.c_double)]
        _lib = L
    return _lib


class OracleError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"oracle: {msg} (status {status})")
        self.status = status


class Oracle:
    """The reference's grouped aggregate restated on the CPU (first-seen group order)."""

    def __init__(self, spec):
        self.spec = spec  # vecruntime_b200.aggregate.Spec (keeps arrays alive)
        self.h = C.c_void_p()
        rc = lib().orc_agg_create(C.byref(spec.spec), C.byref(self.h))
        if rc:
            raise OracleError(rc, lib().orc_last_error().decode())
        n = lib().orc_agg_num_outputs(self.h)
        self.output_types = []
        for i in range(n):
            t = N.ColumnType()
            lib().orc_agg_output_type(self.h, i, C.byref(t))
            self.output_types.append(t)

    def update(self, batch, chunk_rows: int = 4096) -> None:
        cb = batch.ctypes()
        rc = lib().orc_agg_update(self.h, C.byref(cb), chunk_rows)
        if rc:
            raise OracleError(rc, lib().orc_last_error().decode())

    def update_threads(self, batch, threads: int, chunk_rows: int = 4096) -> None:
        """The batch split into `threads` contiguous partitions aggregated on
        that many host threads, then merged here (full-size parity checks)."""
        cb = batch.ctypes()
        rc = lib().orc_agg_update_threads(self.h, C.byref(cb), threads, chunk_rows)
        if rc:
            raise OracleError(rc, lib().orc_last_error().decode())

    def num_groups(self) -> int:
        return lib().orc_agg_num_groups(self.h)

    def key_dictionary(self, key: int):
        """The strings (bytes) behind key `key`'s emitted table ids."""
        n, nb = C.c_int32(), C.c_int64()
        lib().orc_agg_key_dictionary(self.h, key, C.byref(n), None, None, 0, C.byref(nb))
        offs = np.zeros(n.value + 1, np.int32)
        data = np.zeros(max(1, nb.value), np.uint8)
        lib().orc_agg_key_dictionary(self.h, key, C.byref(n), offs.ctypes.data, data.ctypes.data, nb.value,
                                     C.byref(nb))
        return [data[offs[i]:offs[i + 1]].tobytes() for i in range(n.value)]

    def emit(self, fp_mode: int = ORC_FP_COMPENSATED):
        from vecruntime_b200.aggregate import _out_arrays

        n = self.num_groups()
        arrays = [_out_arrays(t, n) for t in self.output_types]
        outs = (N.OutColumn * max(1, len(arrays)))()
        for i, (d, v) in enumerate(arrays):
            outs[i].data = d.ctypes.data
            outs[i].validity = v.ctypes.data
        rc = lib().orc_agg_emit(self.h, 0, n, outs, fp_mode)
        if rc:
            raise OracleError(rc, lib().orc_last_error().decode())
        return arrays

    def close(self):
        if self.h:
            lib().orc_agg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def hash_rows(columns, n: int, finish: bool = True) -> np.ndarray:
    """HashKernels' row hash of host columns (VR_DICT32 keys with their dictionary)."""
    from vecruntime_b200.columns import HostBatch

    types = (N.ColumnType * max(1, len(columns)))(*[c.ctype() for c in columns])
    cb = HostBatch(list(columns), n).ctypes()  # keeps the dictionaries' structs alive
    out = np.zeros(max(n, 1), np.uint32)
    rc = lib().orc_hash_rows(len(columns), types, cb.columns, n, out.ctypes.data, 1 if finish else 0)
    if rc:
        raise OracleError(rc, lib().orc_last_error().decode())
    return out[:n]


def run_threads(spec, batch, threads: int, chunk_rows: int = 4096):
    """Times the oracle on `threads` host threads (one partition each, then
    merged): returns (seconds, groups)."""
    cb = batch.ctypes()
    secs = C.c_double()
    groups = C.c_int64()
    rc = lib().orc_agg_run_threads(C.byref(spec.spec), C.byref(cb), threads, chunk_rows, C.byref(secs),
                                   C.byref(groups))
    if rc:
        raise OracleError(rc, lib().orc_last_error().decode())
    return secs.value, groups.value


# ------------------------------------------------------------------ Parquet pages
def _buf(data: bytes):
    """`data` with 8 bytes of slack after it (the reference tests' segments
    carry the same), as a ctypes buffer."""
    return C.create_string_buffer(bytes(data) + b"\0" * 8, len(data) + 8)


def rle_decode(data: bytes, width: int, n: int) -> np.ndarray:
    """RleBitPackingReader.readInts of n values (uint32)."""
    out = np.zeros(max(n, 1), np.uint32)
    b = _buf(data)
    rc = lib().orc_rle_decode(b, len(data), width, n, out.ctypes.data)
    if rc:
        raise OracleError(rc, lib().orc_pq_last_error().decode())
    return out[:n]


def pq_decode_page(data: bytes, **fields):
    """ParquetPageDecoder.decode of one flat page: (slot bytes, validity
    bitmap bytes, present count); ids for a dictionary page, 0 at a null."""
    page = N.PqPage(None, len(data), **fields)
    vb = 4 if fields.get("encoding") == N.VR_PQ_RLE_DICTIONARY else fields["value_bytes"]
    n = fields["num_values"]
    out = np.zeros(max(n, 1) * vb, np.uint8)
    valid = np.zeros(max(1, (n + 7) // 8), np.uint8)
    present = C.c_int64()
    b = _buf(data)
    rc = lib().orc_pq_decode_page(b, C.byref(page), out.ctypes.data, valid.ctypes.data, C.byref(present))
    if rc:
        raise OracleError(rc, lib().orc_pq_last_error().decode())
    return out[:n * vb], valid[:(n + 7) // 8], present.value


def pq_plain_dictionary(data: bytes, n: int):
    """ParquetPageDecoder.decodeDictionary (BYTE_ARRAY): (offsets, bytes)."""
    total = C.c_int64()
    b = _buf(data)
    rc = lib().orc_pq_plain_dictionary(b, len(data), n, None, None, C.byref(total))
    if rc:
        raise OracleError(rc, lib().orc_pq_last_error().decode())
    offs = np.zeros(n + 1, np.int32)
    out = np.zeros(max(1, total.value), np.uint8)
    rc = lib().orc_pq_plain_dictionary(b, len(data), n, offs.ctypes.data, out.ctypes.data, C.byref(total))
    if rc:
        raise OracleError(rc, lib().orc_pq_last_error().decode())
    return offs, out[:total.value]


def pq_decode_pages_threads(pages, threads: int):
    """Every page of a chunk decoded on `threads` host threads, each into its
    own output (as the reference's decoder returns one buffer set per page):
    (slot bytes of all pages in order, per-page validity bitmaps, seconds)."""
    n = len(pages)
    blobs = [C.create_string_buffer(bytes(b) + b"\0" * 8, len(b) + 8) for b, _ in pages]
    ptrs = (C.c_void_p * max(1, n))(*[C.cast(b, C.c_void_p) for b in blobs])
    descs = (N.PqPage * max(1, n))(*[N.PqPage(None, len(b), **f) for b, f in pages])
    counts = np.array([f["num_values"] for _, f in pages], np.int64)
    vb = 4 if n and pages[0][1]["encoding"] == N.VR_PQ_RLE_DICTIONARY else (pages[0][1]["value_bytes"] if n else 4)
    slot_base = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int64) if n else np.zeros(1, np.int64)
    vbytes = (counts + 7) // 8
    valid_base = np.concatenate([[0], np.cumsum(vbytes)[:-1]]).astype(np.int64) if n else np.zeros(1, np.int64)
    out = np.zeros(max(1, int(counts.sum())) * vb, np.uint8)
    valid = np.zeros(max(1, int(vbytes.sum())), np.uint8)
    secs = C.c_double()
    rc = lib().orc_pq_decode_pages_threads(n, ptrs, descs, slot_base.ctypes.data, valid_base.ctypes.data,
                                           out.ctypes.data, valid.ctypes.data, threads, C.byref(secs))
    if rc:
        raise OracleError(rc, lib().orc_pq_last_error().decode())
    return out[:int(counts.sum()) * vb], valid, secs.value
