"""epi_connect_noalloc: connect_cell for callers that cannot let the library
allocate device memory (their memory belongs to another allocator or a
fixed start-up pool, or their loop must not allocate once running).

The caller owns every buffer (here torch allocates them, as such a caller's
framework would); the entry point itself uses only its fixed device array.
Its lists must equal the reference's frames and the context API's
(epi_get_connections) exactly, call after call, since every call reuses the
same working array. Its two error outputs (count = -1 for a particle outside
the grid, count > max_conn for an overflowed row) are exercised, and the
device's free memory must not change across calls.
"""
import ctypes

import numpy as np
import pytest

from epi_b200 import capi
from epi_b200 import tissue as T
from tests.golden.make_golden import load

pytestmark = pytest.mark.gpu

MAX_PARTICLES = 40960  # EPI_NOALLOC_MAX_PARTICLES
MAX_CONN = 96


def _entry():
    f = capi.lib().epi_connect_noalloc
    f.argtypes = ([ctypes.c_void_p] * 4 + [ctypes.c_int32] * 4 + [ctypes.c_double] * 4 +
                  [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p])
    f.restype = ctypes.c_int
    return f


class _Buffers:
    """Device inputs and outputs of one call, allocated by the caller."""

    def __init__(self, t, max_conn=MAX_CONN):
        import torch
        dev = torch.device("cuda")
        self.t = t
        self.max_conn = max_conn
        self.inputs = [torch.tensor(a, dtype=torch.float64, device=dev)
                       for a in (t.x, t.y, t.z, t.radius)]
        # outputs pre-filled with garbage: every entry that matters must be written
        self.conn = torch.full((t.n, max_conn), -7, dtype=torch.int32, device=dev)
        self.count = torch.full((t.n,), -7, dtype=torch.int32, device=dev)

    def call(self):
        import torch
        t = self.t
        x, y, z, r = self.inputs
        stream = torch.cuda.current_stream().cuda_stream
        rc = _entry()(x.data_ptr(), y.data_ptr(), z.data_ptr(), r.data_ptr(), t.n, t.nmemb,
                      t.nmx, t.nmy, t.lx, t.ly, t.lz, t.params.lj_thresh, self.max_conn,
                      self.conn.data_ptr(), self.count.data_ptr(), stream)
        assert rc == capi.EPI_OK, capi.strerror(rc)
        torch.cuda.synchronize()
        return self.conn.cpu().numpy(), self.count.cpu().numpy()


def _rows(conn, count):
    return np.concatenate([conn[i, :count[i]] for i in range(len(count))])


def _context_lists(t):
    with capi.Context(precision=capi.EPI_PREC_FP64, max_conn=MAX_CONN,
                      max_cand=2 * MAX_CONN) as ctx:
        ctx.upload([t])
        return ctx.connections()


def test_noalloc_lists_equal_reference_and_context_lists_call_after_call(built):
    # consecutive calls on the same device share the working array: a large
    # mixed-state tissue between two small ones must leave no trace
    golden = load("c1")[0]
    for t, frame in ((T.config1(), golden), (T.mixed_state_tissue(), None),
                     (T.config1(9), None), (T.config1(), golden)):
        conn, count = _Buffers(t).call()
        assert count.max() <= MAX_CONN and count.min() >= 0
        off, idx = _context_lists(t)
        assert np.array_equal(count, np.diff(off))
        assert np.array_equal(_rows(conn, count), idx)
        if frame is not None:  # the compiled reference's connect_cell at step 0
            assert np.array_equal(count, np.diff(frame["conn_off"]))
            assert np.array_equal(_rows(conn, count), frame["conn_idx"])


def test_noalloc_allocates_no_device_memory(built):
    import torch
    buf = _Buffers(T.mixed_state_tissue())
    first = buf.call()  # loads the kernels and looks up the working array
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        again = buf.call()
        assert np.array_equal(again[0], first[0]) and np.array_equal(again[1], first[1])
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_marks_a_particle_outside_the_grid(built):
    t = T.config1()
    bad = t.nmemb + 5
    t.z[bad] = t.lz + 8.0  # above the grid: the reference's range assert
    conn, count = _Buffers(t).call()
    assert count[bad] == -1
    ok = np.arange(t.n) != bad
    assert count[ok].min() >= 0
    # no cell's search connected the marked particle; the other rows are the
    # lists of the tissue with that particle far away
    for i in np.nonzero(ok)[0]:
        assert bad not in conn[i, :count[i]]
    far = t.copy()
    far.z[bad] = t.lz - 1.0
    off, idx = _context_lists(far)
    for i in np.nonzero(ok)[0]:
        row = idx[off[i]:off[i + 1]]
        assert np.array_equal(conn[i, :count[i]], row[row != bad])


def test_noalloc_reports_overflowed_rows(built):
    t = T.config1()
    small = 5
    conn, count = _Buffers(t, max_conn=small).call()
    off, idx = _context_lists(t)
    full = np.diff(off)
    assert np.array_equal(count, full)  # the full connected_cell length
    over = count > small
    assert over.any() and (~over).any()
    for i in range(t.n):
        row = idx[off[i]:off[i + 1]]
        if over[i]:  # an unspecified subset of max_conn partners
            assert set(conn[i, :small]) <= set(row) and len(set(conn[i, :small])) == small
        else:
            assert np.array_equal(conn[i, :count[i]], row)


def test_noalloc_rejects_sizes_beyond_its_fixed_array(built):
    f = _entry()
    dummy = 16  # never dereferenced: the size check comes first
    big = f(dummy, dummy, dummy, dummy, MAX_PARTICLES + 1, 0, 0, 0, 16.0, 16.0, 32.0, 1.2,
            MAX_CONN, dummy, dummy, None)
    assert big == capi.EPI_ERR_INVALID_ARG
    # a 128 x 128 x 32 box has 64 * 64 * 16 = 65536 bins, over the 32768 limit
    wide = f(dummy, dummy, dummy, dummy, 1000, 0, 0, 0, 128.0, 128.0, 32.0, 1.2,
             MAX_CONN, dummy, dummy, None)
    assert wide == capi.EPI_ERR_INVALID_ARG
