"""pt_direct_sum_noalloc: the FP64 direct sum for callers that cannot allocate
device memory (their buffers come from their own pool or budget, and
cudaMalloc / cudaFree would also synchronise the whole device).

The test owns every buffer (allocated here with torch) and calls the entry
point through the C ABI twice in a row; both results must match the
allocating entry point, pt_direct_sum, within the direct-sum tolerance the
other tests use.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from paratreet_b200 import ics

pytestmark = pytest.mark.gpu

MAX_TARGETS = (8 * 2 ** 20 - 256) // 8 // 4


def test_direct_sum_noalloc_matches_allocating_entry_point():
    import torch
    from paratreet_b200 import _lib as L
    from paratreet_b200.gravity import GravitySimulation

    p = ics.plummer(20000, seed=21, soft=0.01)
    tgt = np.arange(3, 20000, 5, dtype=np.int32)
    with GravitySimulation() as s:
        s.set_particles(p)
        ref = s.direct_sum(tgt)

    lib = L.load()
    dev = torch.device("cuda", 0)
    src = [torch.from_numpy(np.ascontiguousarray(p[k])).to(dev) for k in ("x", "y", "z", "m", "soft")]
    dtgt = torch.from_numpy(tgt).to(dev)
    outs = [torch.empty(tgt.size, dtype=torch.float64, device=dev) for _ in range(4)]
    err = C.create_string_buffer(256)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    results = []
    for _ in range(2):
        for o in outs:
            o.fill_(float("nan"))
        rc = lib.pt_direct_sum_noalloc(src[0].numel(), *[C.c_void_p(t.data_ptr()) for t in src], tgt.size,
                                       C.c_void_p(dtgt.data_ptr()), *[C.c_void_p(o.data_ptr()) for o in outs],
                                       stream, err, len(err))
        assert rc == 0, err.value.decode()
        results.append([o.cpu().numpy() for o in outs])
    for got in results:
        for a, b in zip(got, ref):
            assert np.all(np.isfinite(a))
            assert np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)) < 1e-12

    # sizes beyond the fixed scratch are refused with a message, before any GPU work
    rc = lib.pt_direct_sum_noalloc(src[0].numel(), *[C.c_void_p(t.data_ptr()) for t in src], MAX_TARGETS + 1,
                                   C.c_void_p(dtgt.data_ptr()), *[C.c_void_p(o.data_ptr()) for o in outs],
                                   stream, err, len(err))
    assert rc == -1 and b"scratch limit" in err.value

    # a target index outside [0, n) is found by the kernel, which skips it (it
    # never reads through a bad index): the call reports it and leaves the
    # outputs untouched, and the next good call starts from a cleared status word
    n = src[0].numel()
    for bad in (n, -1):
        btgt = torch.from_numpy(np.array([0, bad, 7], dtype=np.int32)).to(dev)
        for o in outs:
            o.fill_(float("nan"))
        rc = lib.pt_direct_sum_noalloc(n, *[C.c_void_p(t.data_ptr()) for t in src], 3, C.c_void_p(btgt.data_ptr()),
                                       *[C.c_void_p(o.data_ptr()) for o in outs], stream, err, len(err))
        assert rc == -1 and b"outside [0, n)" in err.value
        assert all(bool(torch.isnan(o[:3]).all()) for o in outs)
    rc = lib.pt_direct_sum_noalloc(n, *[C.c_void_p(t.data_ptr()) for t in src], tgt.size, C.c_void_p(dtgt.data_ptr()),
                                   *[C.c_void_p(o.data_ptr()) for o in outs], stream, err, len(err))
    assert rc == 0, err.value.decode()
    for a, b in zip([o.cpu().numpy() for o in outs], ref):
        assert np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)) < 1e-12
