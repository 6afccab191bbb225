"""Key columns for the row-hash GPU tests: random strings, and host columns
copied to the device as vr_column descriptors (dictionaries included)."""
import ctypes as C

import numpy as np

from vecruntime_b200 import native as N


def device_key_columns(torch, cols, dict_hashes=False):
    """Host key columns copied to the device as vr_column descriptors: data,
    validity, UTF8 offsets, and each dictionary's buffers behind a host
    vr_dictionary (with its entry hashes from vr_hash_dictionary when
    `dict_hashes`). Returns (types, columns, objects to keep alive)."""
    keep = []

    def put(a):
        t = torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).cuda()
        keep.append(t)
        return t.data_ptr()

    types = (N.ColumnType * len(cols))(*[c.ctype() for c in cols])
    dev = (N.Column * len(cols))()
    for i, c in enumerate(cols):
        dev[i].data = put(c.data)
        if c.validity is not None:
            dev[i].validity = put(c.validity)
        if c.offsets is not None:
            dev[i].offsets = put(c.offsets)
        if c.dictionary is not None:
            d = c.dictionary
            nd = N.Dictionary(d.size, 0, put(d.offsets), put(d.data), put(d.validity) if d.validity is not None else None,
                              None)
            if dict_hashes:
                h = torch.empty(max(1, d.size), dtype=torch.int32, device="cuda")
                keep.append(h)
                rc = N.lib().vr_hash_dictionary(C.byref(nd), C.c_void_p(h.data_ptr()),
                                                C.c_void_p(torch.cuda.current_stream().cuda_stream))
                assert rc == N.VR_OK, N.lib().vr_thread_last_error()
                nd.hashes = h.data_ptr()
            keep.append(nd)
            dev[i].dictionary = C.pointer(nd)
    return types, dev, keep


def string_values(rng, n, null_p):
    """Strings of 0..13 bytes (every tail length of hashBytes), some non-ASCII, some null."""
    alphabet = list("abcdefghijklmnopqrstuvwxyz0123456789") + ["é", "ß", "中"]
    out = []
    for _ in range(n):
        if rng.random() < null_p:
            out.append(None)
        else:
            out.append("".join(rng.choice(alphabet, size=int(rng.integers(0, 14)))))
    return out
