"""The allocation-free scoring entry point against rc_score_batch.

rc_score_batch_noalloc is for callers that cannot allocate device memory:
a host application whose device memory belongs to another allocator (a
caching pool that must not be bypassed), or a pipelined search loop on its
own streams, for which cudaMalloc/cudaFree would synchronise the whole
device. The caller passes device buffers; the kernel's scratch is a static
device array. These tests run it twice in a row on the same inputs and check
both results against the context-based rc_score_batch (same objective, same
tolerance as the other scoring tests), cover the programs it refuses (status
3 and NaN for a program deeper than its 16 stack entries) and the malformed
ones (the same status as rc_score_batch), and check that a call made after
rc_score_batch launched the shared scoring kernel with a smaller
shared-memory size still runs. The file is collected last and passes both
alone in a fresh process and after the other tests.
"""
import ctypes
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VAR, ADD, MUL, SIN, HALT = 1, 2, 4, 6, 255


def _deep_program(depth):
    """x0 + (x1 + (x0 + ...)): `depth` pushes before the first add."""
    words = []
    for k in range(depth):
        words += [VAR, k % 2]
    words += [ADD] * (depth - 1) + [HALT]
    return words


def _pack(programs):
    words, off = [], [0]
    for p in programs:
        words += p
        off.append(len(words))
    return np.asarray(words, np.uint32), np.asarray(off, np.uint32)


class _Noalloc:
    """Device copies of one dataset, laid out as the entry point wants."""

    def __init__(self, x, y):
        import torch
        v, n = x.shape
        self.n, self.v = n, v
        self.ld = ((n + 1023) // 1024) * 1024
        cols = np.zeros((v, self.ld), np.float32)
        cols[:, :n] = x
        yy = np.zeros(self.ld, np.float32)
        yy[:n] = y
        self.cols = torch.from_numpy(cols).cuda()
        self.y = torch.from_numpy(yy).cuda()

    def score(self, L, prog, off, kind):
        import torch
        P = len(off) - 1
        d_prog = torch.from_numpy(prog.astype(np.int64).astype(np.int32)).cuda()
        d_off = torch.from_numpy(off.astype(np.int32)).cuda()
        d_out = torch.full((P,), -1.0, dtype=torch.float64, device="cuda")
        d_status = torch.full((P,), -1, dtype=torch.int32, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        rc = L.rc_score_batch_noalloc(self.cols.data_ptr(), self.y.data_ptr(), self.n, self.v,
                                      self.ld, d_prog.data_ptr(), d_off.data_ptr(), P, kind,
                                      d_out.data_ptr(), d_status.data_ptr(),
                                      ctypes.c_void_p(stream))
        torch.cuda.synchronize()
        return rc, d_out.cpu().numpy(), d_status.cpu().numpy()


def _check(out, status, want, want_status, tag):
    assert np.array_equal(status, want_status), tag
    ok = status == 0
    tol = 1e-12 * (1.0 + np.abs(want[ok]))
    assert np.all(np.abs(out[ok] - want[ok]) <= tol), tag
    assert np.all(np.isinf(out[status == 2])), tag


def test_noalloc_matches_score_batch_twice(pkg):
    W = importlib.import_module("the-rule-and-compass_b200.workloads")
    dev = importlib.import_module("the-rule-and-compass_b200.device")
    L = dev.lib()
    P, n, v = 300, 20000, 5
    trees, x, y = W.scoring_workload(P, n, seed=21)
    prog, off = pkg.Population(trees).programs()

    ev = pkg.GpuEvaluator(x.reshape(-1), n, v, y)
    ref = {k: ev.score_batch(prog, off, k)[:2] for k in range(5)}
    ev.close()

    na = _Noalloc(x, y)
    for kind in range(5):
        for call in range(2):
            rc, out, status = na.score(L, prog, off, kind)
            assert rc == 0
            _check(out, status, *ref[kind], (kind, call))
            if kind != 4:
                assert (status == 0).sum() > P // 4


def test_noalloc_refuses_deep_programs_and_flags_malformed_ones(pkg):
    """A program deeper than 16 stack entries is refused with status 3 and
    NaN (rc_score_batch scores it); truncated, underflowing, unterminated and
    unknown-opcode programs get rc_score_batch's status."""
    W = importlib.import_module("the-rule-and-compass_b200.workloads")
    dev = importlib.import_module("the-rule-and-compass_b200.device")
    L = dev.lib()
    n, v = 9000, 5
    trees, x, y = W.scoring_workload(40, n, seed=5)
    good_prog, good_off = pkg.Population(trees).programs()
    programs = [list(good_prog[good_off[i]:good_off[i + 1]]) for i in range(40)]
    deep = [4, 7, 12]
    programs[deep[0]] = _deep_program(18)
    programs[deep[1]] = _deep_program(24)
    programs[deep[2]] = _deep_program(40)
    programs[33] = [MUL] + _deep_program(20)      # underflow before a deep stack
    programs[20] = [VAR, 0, VAR]                 # truncated operand
    programs[21] = [VAR, 0, ADD, HALT]           # stack underflow
    programs[22] = [VAR, 1, SIN]                 # no HALT
    programs[23] = [VAR, 0, 200, HALT]           # unknown opcode
    programs[24] = [VAR, 9, HALT]                # input index out of range
    programs[25] = _deep_program(16)             # 16 entries: still accepted
    prog, off = _pack(programs)

    ev = pkg.GpuEvaluator(x.reshape(-1), n, v, y)
    want, want_status = ev.score_batch(prog, off, 0)[:2]
    ev.close()

    na = _Noalloc(x, y)
    for call in range(2):
        rc, out, status = na.score(L, prog, off, 0)
        assert rc == 0
        for k in deep:
            assert status[k] == 3 and np.isnan(out[k]), (call, k, status[k], out[k])
            assert want_status[k] == 0, "rc_score_batch scores deep programs"
        keep = np.ones(len(programs), bool)
        keep[deep] = False
        _check(out[keep], status[keep], want[keep], want_status[keep], call)
        assert status[25] == 0


def test_noalloc_after_score_batch_with_deep_spills(pkg):
    """rc_score_batch launches the shared scoring kernel with the shared
    memory its bucket needs (8 or more spill slots here). A later call of the
    allocation-free entry point, which needs more, must still run and match."""
    W = importlib.import_module("the-rule-and-compass_b200.workloads")
    dev = importlib.import_module("the-rule-and-compass_b200.device")
    L = dev.lib()
    n, v = 12000, 5
    trees, x, y = W.scoring_workload(64, n, seed=9)
    prog, off = pkg.Population(trees).programs()
    spill = _pack([_deep_program(d) for d in (10, 11, 12, 13)])

    ev = pkg.GpuEvaluator(x.reshape(-1), n, v, y)
    want, want_status = ev.score_batch(prog, off, 0)[:2]
    na = _Noalloc(x, y)
    rc, out, status = na.score(L, prog, off, 0)
    assert rc == 0
    _check(out, status, want, want_status, "before")
    sw, ss = ev.score_batch(spill[0], spill[1], 0)[:2]
    assert np.all(ss == 0), ss
    for call in range(2):
        rc, out, status = na.score(L, prog, off, 0)
        assert rc == 0, call
        _check(out, status, want, want_status, ("after", call))
    rc, out, status = na.score(L, spill[0], spill[1], 0)
    assert rc == 0
    _check(out, status, sw, ss, "spill programs")
    ev.close()


def test_noalloc_rejects_oversized_batches(pkg):
    import torch
    dev = importlib.import_module("the-rule-and-compass_b200.device")
    L = dev.lib()
    n, v, P = 1 << 20, 5, 100000  # ~200 MB of decoded programs: beyond the 16 MiB scratch
    d = torch.zeros(16, dtype=torch.float32, device="cuda")
    rc = L.rc_score_batch_noalloc(d.data_ptr(), d.data_ptr(), n, v, n, d.data_ptr(),
                                  d.data_ptr(), P, 0, d.data_ptr(), d.data_ptr(), None)
    assert rc == -2
