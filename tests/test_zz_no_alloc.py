"""The allocation-free scoring entry point against rc_score_batch.

rc_score_batch_noalloc is for callers that cannot allocate device memory
(their device memory belongs to another allocator, or cudaMalloc's implicit
device synchronisation would stall their pipelined streams). The caller
passes device buffers; the kernel's scratch is a static device array. This
test runs it twice in a row on the same inputs and checks both results
against the context-based rc_score_batch (same objective, same tolerance as
the other scoring tests). It sits in its own file, collected last, and must
pass both alone in a fresh process and after the other tests.
"""
import ctypes
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_score_batch_twice(pkg):
    import torch
    W = importlib.import_module("the-rule-and-compass_b200.workloads")
    dev = importlib.import_module("the-rule-and-compass_b200.device")
    L = dev.lib()
    P, n, v = 300, 20000, 5
    trees, x, y = W.scoring_workload(P, n, seed=21)
    prog, off = pkg.Population(trees).programs()

    ev = pkg.GpuEvaluator(x.reshape(-1), n, v, y)
    ref = {k: ev.score_batch(prog, off, k)[:2] for k in (0, 1)}
    ev.close()

    ld = ((n + 1023) // 1024) * 1024
    cols_h = np.zeros((v, ld), np.float32)
    cols_h[:, :n] = x
    y_h = np.zeros(ld, np.float32)
    y_h[:n] = y
    d_cols = torch.from_numpy(cols_h).cuda()
    d_y = torch.from_numpy(y_h).cuda()
    d_prog = torch.from_numpy(prog.astype(np.int32)).cuda()
    d_off = torch.from_numpy(off.astype(np.int32)).cuda()
    d_out = torch.zeros(P, dtype=torch.float64, device="cuda")
    d_status = torch.zeros(P, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for kind in (0, 1):
        for call in range(2):
            d_out.fill_(-1.0)
            d_status.fill_(-1)
            rc = L.rc_score_batch_noalloc(d_cols.data_ptr(), d_y.data_ptr(), n, v, ld,
                                          d_prog.data_ptr(), d_off.data_ptr(), P, kind,
                                          d_out.data_ptr(), d_status.data_ptr(),
                                          ctypes.c_void_p(stream))
            assert rc == 0
            torch.cuda.synchronize()
            out = d_out.cpu().numpy()
            status = d_status.cpu().numpy()
            want, want_status = ref[kind]
            assert np.array_equal(status, want_status), (kind, call)
            ok = status == 0
            assert ok.sum() > P // 4
            tol = 1e-12 * (1.0 + np.abs(want[ok]))
            assert np.all(np.abs(out[ok] - want[ok]) <= tol), (kind, call)
            assert np.all(np.isinf(out[~ok]))


def test_noalloc_rejects_oversized_batches(pkg):
    import torch
    dev = importlib.import_module("the-rule-and-compass_b200.device")
    L = dev.lib()
    n, v, P = 1 << 20, 5, 100000  # ~200 MB of decoded programs: beyond the 16 MiB scratch
    d = torch.zeros(16, dtype=torch.float32, device="cuda")
    rc = L.rc_score_batch_noalloc(d.data_ptr(), d.data_ptr(), n, v, n, d.data_ptr(),
                                  d.data_ptr(), P, 0, d.data_ptr(), d.data_ptr(), None)
    assert rc == -2
