"""Arrow-layout columns and batches on the host (numpy) or on the device.

Layout follows the reference's VectorBuffers contract
(kernels/src/main/java/io/vecruntime/kernels/VectorBuffers.java:23-67):
little-endian values, LSB-first validity bitmap (None = all valid),
DECIMAL128 as two little-endian int64 limbs per value (Decimal128.java:21-61),
BOOL bit-packed.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

import ctypes as C

from . import native as N

LANE_NAMES = {N.VR_INT32: "INT32", N.VR_INT64: "INT64", N.VR_FLOAT64: "FLOAT64", N.VR_BOOL: "BOOL",
              N.VR_DECIMAL128: "DECIMAL128", N.VR_DICT32: "DICT32", N.VR_UTF8: "UTF8"}


def pack_bits(mask) -> np.ndarray:
    """bool array -> LSB-first bitmap (uint8), padded to a multiple of 8 bytes."""
    mask = np.asarray(mask, dtype=bool)
    b = np.packbits(mask, bitorder="little")
    pad = (-len(b)) % 8
    if pad:
        b = np.concatenate([b, np.zeros(pad, np.uint8)])
    return b


def unpack_bits(bm: np.ndarray, n: int) -> np.ndarray:
    return np.unpackbits(np.asarray(bm, dtype=np.uint8), bitorder="little", count=n).astype(bool)


def dec128_from_ints(values: Sequence[int]) -> np.ndarray:
    """Python ints -> (n, 2) uint64 limbs (lo, hi), two's complement."""
    out = np.zeros((len(values), 2), dtype=np.uint64)
    for i, v in enumerate(values):
        u = int(v) & ((1 << 128) - 1)
        out[i, 0] = u & 0xFFFFFFFFFFFFFFFF
        out[i, 1] = u >> 64
    return out


def dec128_to_ints(limbs: np.ndarray) -> List[int]:
    out = []
    for lo, hi in np.asarray(limbs, dtype=np.uint64).reshape(-1, 2):
        u = (int(hi) << 64) | int(lo)
        out.append(u - (1 << 128) if u >> 127 else u)
    return out


def _utf8_buffers(values):
    """bytes/str values (None for a null) -> (int32 offsets, uint8 data, null mask)."""
    raw = [b"" if v is None else (v.encode() if isinstance(v, str) else bytes(v)) for v in values]
    offsets = np.zeros(len(raw) + 1, np.int32)
    offsets[1:] = np.cumsum([len(b) for b in raw])
    data = np.frombuffer(b"".join(raw) + b"\0" * 16, np.uint8).copy()  # padded: never empty
    return offsets, data, np.array([v is None for v in values], bool)


@dataclass
class Dictionary:
    """An Arrow string dictionary (the values a VR_DICT32 column's ids point
    into): int32 offsets, UTF-8 bytes, optional entry validity. A null entry
    makes the rows that point at it null (GroupKeyTable.java:1388-1389)."""
    offsets: np.ndarray
    data: np.ndarray
    validity: Optional[np.ndarray] = None
    hashes: Optional[np.ndarray] = None  # hashBytes per entry, optional

    @property
    def size(self) -> int:
        return len(self.offsets) - 1

    def ctypes(self) -> N.Dictionary:
        return N.Dictionary(self.size, 0, self.offsets.ctypes.data, self.data.ctypes.data,
                            self.validity.ctypes.data if self.validity is not None else None,
                            self.hashes.ctypes.data if self.hashes is not None else None)


def dictionary(entries) -> Dictionary:
    """A dictionary from str/bytes entries (None = a null entry)."""
    offsets, data, nulls = _utf8_buffers(entries)
    return Dictionary(offsets, data, pack_bits(~nulls) if nulls.any() else None)


@dataclass
class Col:
    """One input column: lane type, values and optional validity bitmap;
    VR_UTF8 adds its offsets, VR_DICT32 may carry its dictionary."""
    lane: int
    data: np.ndarray
    validity: Optional[np.ndarray] = None
    precision: int = 0
    scale: int = 0
    dict_size: int = 0
    nullable: Optional[bool] = None
    offsets: Optional[np.ndarray] = None
    dictionary: Optional[Dictionary] = None

    @property
    def length(self) -> int:
        if self.lane == N.VR_BOOL:
            return self._n
        return len(self.data)

    def ctype(self) -> N.ColumnType:
        """The column's type in a spec; a VR_DICT32 column that carries a
        dictionary declares that its batches bring their own."""
        nullable = self.validity is not None if self.nullable is None else self.nullable
        flags = N.VR_COL_BATCH_DICTIONARY if (self.lane == N.VR_DICT32 and self.dictionary is not None) else 0
        return N.ColumnType(self.lane, self.precision, self.scale, 1 if nullable else 0, self.dict_size, flags)


def _validity(nulls, n):
    if nulls is None:
        return None
    nulls = np.asarray(nulls, dtype=bool)
    assert len(nulls) == n
    return pack_bits(~nulls)


def ints(values, nulls=None, **kw) -> Col:
    v = np.ascontiguousarray(values, dtype=np.int32)
    return Col(N.VR_INT32, v, _validity(nulls, len(v)), **kw)


def longs(values, nulls=None, **kw) -> Col:
    v = np.ascontiguousarray(values, dtype=np.int64)
    return Col(N.VR_INT64, v, _validity(nulls, len(v)), **kw)


def doubles(values, nulls=None, **kw) -> Col:
    v = np.ascontiguousarray(values, dtype=np.float64)
    return Col(N.VR_FLOAT64, v, _validity(nulls, len(v)), **kw)


def decimals(unscaled, precision, scale, nulls=None, **kw) -> Col:
    """DECIMAL(p <= 18, s) as an INT64 lane of unscaled values (TypeMapping.java:87-90)."""
    v = np.ascontiguousarray(unscaled, dtype=np.int64)
    return Col(N.VR_INT64, v, _validity(nulls, len(v)), precision=precision, scale=scale, **kw)


def decimals128(values, precision, scale, nulls=None, **kw) -> Col:
    v = dec128_from_ints(values)
    return Col(N.VR_DECIMAL128, v, _validity(nulls, len(v)), precision=precision, scale=scale, **kw)


def dict_ids(ids, dict_size, nulls=None, **kw) -> Col:
    """A dictionary-encoded UTF8 key as table-level dictionary ids."""
    v = np.ascontiguousarray(ids, dtype=np.int32)
    return Col(N.VR_DICT32, v, _validity(nulls, len(v)), dict_size=dict_size, **kw)


def strings(values, **kw) -> Col:
    """A plain UTF8 column from str/bytes values (None = null)."""
    offsets, data, nulls = _utf8_buffers(values)
    return Col(N.VR_UTF8, data, pack_bits(~nulls) if nulls.any() else None, offsets=offsets, **kw)


def dict_strings(ids, dict_: Dictionary, nulls=None, **kw) -> Col:
    """A dictionary-encoded UTF8 column: ids into `dict_`, carried with it."""
    v = np.ascontiguousarray(ids, dtype=np.int32)
    return Col(N.VR_DICT32, v, _validity(nulls, len(v)), dictionary=dict_, **kw)


def bools(values, nulls=None, **kw) -> Col:
    b = np.asarray(values, dtype=bool)
    c = Col(N.VR_BOOL, pack_bits(b), _validity(nulls, len(b)), dict_size=2, **kw)
    c._n = len(b)
    return c


@dataclass
class HostBatch:
    """A batch of host columns, kept alive while a ctypes view exists."""
    columns: List[Col]
    num_rows: int
    selection: Optional[np.ndarray] = None  # bitmap
    _keep: list = field(default_factory=list)

    def ctypes(self) -> N.Batch:
        arr = (N.Column * max(1, len(self.columns)))()
        keep = [arr]
        for i, c in enumerate(self.columns):
            arr[i].data = c.data.ctypes.data if c.data is not None and c.data.size else None
            arr[i].validity = c.validity.ctypes.data if c.validity is not None else None
            arr[i].offsets = c.offsets.ctypes.data if c.offsets is not None else None
            if c.dictionary is not None:
                d = c.dictionary.ctypes()
                keep.append(d)
                arr[i].dictionary = C.pointer(d)
        self._keep = keep
        sel = self.selection.ctypes.data if self.selection is not None else None
        return N.Batch(self.num_rows, arr, sel, N.VR_HOST, 0)


def host_batch(columns: List[Col], selection=None) -> HostBatch:
    n = columns[0].length if columns else 0
    sel = pack_bits(selection) if selection is not None and np.asarray(selection).dtype == bool else selection
    return HostBatch(list(columns), n, sel)


@dataclass
class DeviceBatch:
    """Device-resident columns as raw device pointers (e.g. torch tensors'
    data_ptr); `dictionaries`: per column an N.Dictionary of device buffers, or None."""
    num_rows: int
    data_ptrs: List[int]
    validity_ptrs: List[Optional[int]]
    selection_ptr: Optional[int] = None
    dictionaries: Optional[list] = None
    _keep: list = field(default_factory=list)

    def ctypes(self) -> N.Batch:
        arr = (N.Column * max(1, len(self.data_ptrs)))()
        keep = [arr]
        for i, (d, v) in enumerate(zip(self.data_ptrs, self.validity_ptrs)):
            arr[i].data = d
            arr[i].validity = v
            if self.dictionaries and self.dictionaries[i] is not None:
                keep.append(self.dictionaries[i])
                arr[i].dictionary = C.pointer(self.dictionaries[i])
        self._keep = keep
        return N.Batch(self.num_rows, arr, self.selection_ptr, N.VR_DEVICE, 0)


def to_device(batch: HostBatch, device: int = 0):
    """Copies a host batch to the device with torch (plumbing only); returns
    (DeviceBatch, tensors) -- keep `tensors` alive while the batch is used."""
    import torch

    dev = torch.device("cuda", device)
    tensors = []

    def put(a):
        if a is None:
            return None
        # pad to 16 bytes so whole 4-byte words and bulk copies stay inside the buffer
        raw = np.frombuffer(np.ascontiguousarray(a).tobytes(), dtype=np.uint8)
        pad = (-len(raw)) % 16
        if pad:
            raw = np.concatenate([raw, np.zeros(pad, np.uint8)])
        t = torch.from_numpy(raw.copy()).to(dev)
        tensors.append(t)
        return t.data_ptr()

    d = [put(c.data) for c in batch.columns]
    v = [put(c.validity) for c in batch.columns]
    s = put(batch.selection)
    dicts = None
    if any(c.dictionary is not None for c in batch.columns):
        dicts = []
        for c in batch.columns:
            if c.dictionary is None:
                dicts.append(None)
                continue
            dd = c.dictionary
            dicts.append(N.Dictionary(dd.size, 0, put(dd.offsets), put(dd.data), put(dd.validity), None))
    return DeviceBatch(batch.num_rows, d, v, s, dicts), tensors
