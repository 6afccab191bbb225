"""vr_hash_rows_noalloc (descriptors in the library's fixed device scratch)
against vr_hash_rows (descriptors in cudaMalloc'd memory): the same hashes,
call after call. Collected last so it also runs after every other GPU test."""
import ctypes as C

import numpy as np
import pytest

from vecruntime_b200 import native as N

pytestmark = pytest.mark.gpu


def key_columns(torch, rng, n, lanes):
    """Device key columns of the given lanes, every other one with nulls;
    returns (types, columns, tensors kept alive)."""
    types = (N.ColumnType * len(lanes))()
    cols = (N.Column * len(lanes))()
    keep = []
    for i, lane in enumerate(lanes):
        if lane == N.VR_INT32:
            data = torch.from_numpy(rng.integers(-1000, 1000, n, dtype=np.int32)).cuda()
        elif lane in (N.VR_INT64, N.VR_FLOAT64):
            data = torch.from_numpy(rng.integers(-(1 << 62), 1 << 62, n, dtype=np.int64)).cuda()
        elif lane == N.VR_DECIMAL128:
            data = torch.from_numpy(rng.integers(-(1 << 62), 1 << 62, 2 * n, dtype=np.int64)).cuda()
        else:
            data = torch.from_numpy(rng.integers(0, 256, (n + 7) // 8, dtype=np.uint8)).cuda()
        nullable = i % 2 == 1
        valid = torch.from_numpy(rng.integers(0, 256, (n + 7) // 8, dtype=np.uint8)).cuda() if nullable else None
        types[i].lane = lane
        types[i].precision = 38 if lane == N.VR_DECIMAL128 else 0
        types[i].nullable = int(nullable)
        cols[i].data = data.data_ptr()
        cols[i].validity = valid.data_ptr() if nullable else None
        keep += [data, valid]
    return types, cols, keep


def test_noalloc_hashes_match_the_allocating_entry_point_on_two_calls_in_a_row(cuda):
    torch = cuda
    L = N.lib()
    rng = np.random.default_rng(20261203)
    stream = torch.cuda.current_stream().cuda_stream
    cases = [(100_003, [N.VR_INT64, N.VR_INT32, N.VR_DECIMAL128], 1),
             (4_099, [N.VR_BOOL, N.VR_FLOAT64, N.VR_INT32, N.VR_INT64, N.VR_DECIMAL128], 0)]
    # both calls enqueued back to back before anything is read back
    results = []
    for n, lanes, finish in cases:
        types, cols, keep = key_columns(torch, rng, n, lanes)
        out = torch.empty(n, dtype=torch.int32, device="cuda")
        rc = L.vr_hash_rows_noalloc(len(lanes), types, cols, n, C.c_void_p(out.data_ptr()), finish, C.c_void_p(stream))
        assert rc == N.VR_OK, L.vr_thread_last_error()
        results.append((n, lanes, finish, types, cols, keep, out))
    for n, lanes, finish, types, cols, keep, out in results:
        want = torch.empty(n, dtype=torch.int32, device="cuda")
        rc = L.vr_hash_rows(len(lanes), types, cols, n, C.c_void_p(want.data_ptr()), finish, C.c_void_p(stream))
        assert rc == N.VR_OK, L.vr_thread_last_error()
        torch.cuda.synchronize()
        assert torch.equal(out, want), f"{lanes}: noalloc hashes differ"


def test_noalloc_dictionary_keys_match_the_allocating_entry_point(cuda):
    """Dictionary strings: the caller brings the entries' hashes (computed
    once per dictionary with vr_hash_dictionary into its own buffer), since
    this entry point has no room for them; both calls in a row agree with
    vr_hash_rows, which computes them itself. Without the hashes the call is
    refused before anything is enqueued."""
    from keycols import device_key_columns, string_values
    from vecruntime_b200 import columns as Cc

    torch = cuda
    L = N.lib()
    rng = np.random.default_rng(7)
    stream = torch.cuda.current_stream().cuda_stream
    outs = []
    for n in (20_011, 513):
        entries = string_values(rng, 97, 0.02)
        cols = [Cc.dict_strings(rng.integers(0, 97, n), Cc.dictionary(entries), rng.random(n) < 0.1, nullable=True),
                Cc.longs(rng.integers(-(1 << 62), 1 << 62, n, dtype=np.int64))]
        types, dev, keep = device_key_columns(torch, cols, dict_hashes=True)
        out = torch.empty(n, dtype=torch.int32, device="cuda")
        rc = L.vr_hash_rows_noalloc(2, types, dev, n, C.c_void_p(out.data_ptr()), 1, C.c_void_p(stream))
        assert rc == N.VR_OK, L.vr_thread_last_error()
        outs.append((n, cols, types, dev, keep, out))
    for n, cols, types, dev, keep, out in outs:
        plain_types, plain_dev, plain_keep = device_key_columns(torch, cols, dict_hashes=False)
        want = torch.empty(n, dtype=torch.int32, device="cuda")
        rc = L.vr_hash_rows(2, plain_types, plain_dev, n, C.c_void_p(want.data_ptr()), 1, C.c_void_p(stream))
        assert rc == N.VR_OK, L.vr_thread_last_error()
        torch.cuda.synchronize()
        assert torch.equal(out, want), "noalloc dictionary hashes differ"
        rc = L.vr_hash_rows_noalloc(2, plain_types, plain_dev, n, C.c_void_p(out.data_ptr()), 1, C.c_void_p(stream))
        assert rc == N.VR_ERR_INVALID and b"hashes" in L.vr_thread_last_error()


def test_noalloc_refuses_more_keys_than_its_scratch_holds(cuda):
    torch = cuda
    L = N.lib()
    types = (N.ColumnType * 17)()
    cols = (N.Column * 17)()
    out = torch.empty(8, dtype=torch.int32, device="cuda")
    rc = L.vr_hash_rows_noalloc(17, types, cols, 8, C.c_void_p(out.data_ptr()), 1, None)
    assert rc == N.VR_ERR_INVALID
    assert b"scratch" in L.vr_thread_last_error()
