"""epi_connect_noalloc: connect_cell for callers that cannot let the library
allocate device memory (their memory belongs to another allocator or a
fixed start-up pool, or their loop must not allocate once running).

The caller owns every buffer (here torch allocates them, as such a caller's
framework would); the entry point itself uses only its fixed device array.
Its lists must equal the context API's (epi_get_connections) exactly, call
after call, since every call reuses the same working array.
"""
import ctypes

import numpy as np
import pytest

from epi_b200 import capi
from epi_b200 import tissue as T

pytestmark = pytest.mark.gpu

MAX_PARTICLES = 40960  # EPI_NOALLOC_MAX_PARTICLES
MAX_CONN = 96


def _entry():
    f = capi.lib().epi_connect_noalloc
    f.argtypes = ([ctypes.c_void_p] * 4 + [ctypes.c_int32] * 4 + [ctypes.c_double] * 4 +
                  [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p])
    f.restype = ctypes.c_int
    return f


def _noalloc_lists(t):
    import torch
    dev = torch.device("cuda")
    x, y, z, r = (torch.tensor(a, dtype=torch.float64, device=dev)
                  for a in (t.x, t.y, t.z, t.radius))
    # outputs pre-filled with garbage: every entry that matters must be written
    conn = torch.full((t.n, MAX_CONN), -7, dtype=torch.int32, device=dev)
    count = torch.full((t.n,), -7, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    rc = _entry()(x.data_ptr(), y.data_ptr(), z.data_ptr(), r.data_ptr(), t.n, t.nmemb, t.nmx,
                  t.nmy, t.lx, t.ly, t.lz, t.params.lj_thresh, MAX_CONN, conn.data_ptr(),
                  count.data_ptr(), stream)
    assert rc == capi.EPI_OK, capi.strerror(rc)
    torch.cuda.synchronize()
    return conn.cpu().numpy(), count.cpu().numpy()


def _context_lists(t):
    with capi.Context(precision=capi.EPI_PREC_FP64, max_conn=MAX_CONN,
                      max_cand=2 * MAX_CONN) as ctx:
        ctx.upload([t])
        return ctx.connections()


def test_noalloc_lists_equal_context_lists_call_after_call(built):
    # consecutive calls on the same device share the working array: a large
    # mixed-state tissue between two small ones must leave no trace
    for t in (T.config1(), T.mixed_state_tissue(), T.config1(9)):
        conn, count = _noalloc_lists(t)
        off, idx = _context_lists(t)
        assert np.array_equal(count, np.diff(off))
        assert count.max() <= MAX_CONN and count.min() >= 0
        rows = np.concatenate([conn[i, :count[i]] for i in range(t.n)])
        assert np.array_equal(rows, idx)


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
