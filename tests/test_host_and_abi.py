"""Host-side compiler and C-ABI surface (CPU only, no device calls).

Restates the reference's host tests: emitted words (my-version/src/gpu.rs:
349-438), the stack guard and lowering (gpu.rs:3402-3438), the fit-plan cap
and rejection labels (gpu.rs:4554-4598, fit.rs:958-1056). The ABI test loads
librcsr_b200.so and checks that it exports every function include/rcsr_b200.h
declares.
"""
import ctypes
import importlib
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def f32bits(v):
    return int(np.float32(v).view(np.uint32))


def test_emitted_words(pkg, E):
    t = E.node(E.ADD, [E.node(E.MUL, [E.input(0), E.constant(2.0)]), E.constant(1.0)])
    words, lowered = pkg.compile_program(t)
    assert list(words) == [1, 0, 0, f32bits(2.0), 4, 0, f32bits(1.0), 2, 255]
    assert not lowered


def test_constants_are_rounded_to_f32(pkg, E):
    words, _ = pkg.compile_program(E.constant(0.1))
    assert list(words) == [0, f32bits(0.1), 255]


def test_lowering_rewrites_inverse_hyperbolics(pkg, E, O):
    for op in (E.ASINH, E.ACOSH, E.ATANH):
        t = E.node(op, [E.input(0)])
        words, lowered = pkg.compile_program(t)
        assert lowered
        assert 64 not in words and 65 not in words and 66 not in words


def test_stack_guard(pkg, E):
    deep = E.input(0)
    for _ in range(56):
        deep = E.node(E.ADD, [E.input(1), deep])
    assert pkg.host.peak_stack(deep) > 56
    with pytest.raises(pkg.host.CompileError):
        pkg.compile_program(deep)
    pop = pkg.Population([deep, E.input(0)])
    assert len(pop) == 1 and pop.unsupported == 1


def test_population_offsets(pkg, E):
    trees = [E.input(0), E.node(E.SIN, [E.input(1)]), E.constant(3.0)]
    pop = pkg.Population(trees)
    prog, off = pop.programs()
    assert list(off) == [0, 3, 7, 10]
    assert len(prog) == 10


def test_fit_plan_records(pkg, E):
    # c0 * x0 + c1: post-order [const, var, mul, const, add]
    t = E.node(E.ADD, [E.node(E.MUL, [E.constant(1.5), E.input(0)]), E.constant(-0.5)])
    plan = pkg.gpu_fit_plan(t)
    assert plan.nconst == 2
    assert list(plan.c0) == [1.5, -0.5]
    rec = plan.words.reshape(-1, 4)
    assert [list(r) for r in rec] == [[0, 0, 0, 0], [1, 0, 0, 0], [4, 0, 1, 0xFFFFFFFF],
                                      [0, 0, 0, 1], [2, 2, 3, 0xFFFFFFFF]]
    # the correlation gauge: Add(Mul(Const, T), Const) -> (scale, offset)
    assert list(plan.gauge) == [0, 1]


def test_fit_plan_cap_and_rejections(pkg, E):
    for p in range(1, 21):
        terms = [E.node(E.MUL, [E.constant(0.1), E.input(k)]) for k in range(p)]
        t = terms.pop()
        while terms:
            t = E.node(E.ADD, [terms.pop(), t])
        assert pkg.gpu_fit_plan(t).nconst == p
    t = E.node(E.ADD, [t, E.constant(1.0)])
    with pytest.raises(pkg.host.GpuFitReject) as e:
        pkg.gpu_fit_plan(t)
    assert e.value.label == "too_many_constants"
    with pytest.raises(pkg.host.GpuFitReject) as e:
        pkg.gpu_fit_plan(E.node(E.SIN, [E.input(0)]))
    assert e.value.label == "no_constants"
    with pytest.raises(pkg.host.GpuFitReject) as e:
        pkg.gpu_fit_plan(E.node(E.FLOOR, [E.node(E.MUL, [E.constant(2.0), E.input(0)])]))
    assert e.value.label == "unsupported_op"


def _declared_functions():
    src = open(os.path.join(ROOT, "include", "rcsr_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(rc_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(pkg):
    path = os.path.join(ROOT, "the-rule-and-compass_b200", "librcsr_b200.so")
    assert os.path.exists(path), "build the CUDA library first"
    lib = ctypes.CDLL(path)
    names = _declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers the same surface
    from importlib import import_module
    dev = import_module("the-rule-and-compass_b200.device")
    assert sorted(dev.SIGNATURES) == names


def test_host_library_exports_every_refit_symbol(pkg):
    """include/rcsr_refit.h is served by librcsr_host.so (no GPU needed)."""
    src = open(os.path.join(ROOT, "include", "rcsr_refit.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = sorted(set(re.findall(r"\b(rch_[a-z0-9_]+)\s*\(", src)))
    assert names == ["rch_refit_finalists", "rch_soa_eval", "rch_soa_sse"]
    lib = ctypes.CDLL(os.path.join(ROOT, "the-rule-and-compass_b200", "librcsr_host.so"))
    assert all(hasattr(lib, n) for n in names)


def test_host_library_exports_every_host_symbol(pkg):
    """include/rcsr_host.h (the compiler, fit plans, admission, constant
    write-back) is served by librcsr_host.so."""
    src = open(os.path.join(ROOT, "include", "rcsr_host.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = sorted(set(re.findall(r"\b(rch_[a-z0-9_]+)\s*\(", src)))
    assert len(names) == 9, names
    lib = ctypes.CDLL(os.path.join(ROOT, "the-rule-and-compass_b200", "librcsr_host.so"))
    assert all(hasattr(lib, n) for n in names), [n for n in names if not hasattr(lib, n)]


def test_fit_kernel_info_contract(pkg):
    L = pkg.cuda_lib()
    t, s, m = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    assert L.rc_fit_kernel_info(20, ctypes.byref(t), ctypes.byref(s), ctypes.byref(m)) == 0
    assert m.value == 20 and t.value > 0 and s.value > 0
    assert L.rc_fit_kernel_info(21, ctypes.byref(t), ctypes.byref(s), ctypes.byref(m)) == -1


def test_rank_method_switch_refuses_bad_arguments(pkg):
    """rc_rank_tuning and rc_rank_last_fallbacks return -1 on a null context
    (no device needed)."""
    L = pkg.cuda_lib()
    L.rc_rank_tuning.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    L.rc_rank_last_fallbacks.argtypes = [ctypes.c_void_p]
    assert L.rc_rank_tuning(None, 0, 0) == -1
    assert L.rc_rank_last_fallbacks(None) == -1


def test_fit_admission_rules(pkg):
    """search.rs:3006-3074: admission_count and select_promoted."""
    H = importlib.import_module("the-rule-and-compass_b200.host")
    assert H.admission_count(100, 1000) == 32
    assert H.admission_count(200, 1000) == 50
    assert H.admission_count(20, 1000) == 20
    assert H.admission_count(1000, 1 << 20) == 1000
    assert H.admission_count(0, 10) == 1
    rng = np.random.Generator(np.random.PCG64(5))
    pops = [40, 200, 7]
    pending = [(i, j) for i, p in enumerate(pops) for j in range(p) if rng.uniform() < 0.8]
    err = np.round(rng.uniform(0, 1, len(pending)), 1)      # many ties
    cx = rng.integers(1, 5, len(pending)).astype(float)       # ties too
    hc = rng.uniform(size=len(pending)) < 0.9
    for rows in (1000, 1 << 20):
        got = H.select_promoted(pops, pending, err, cx, hc, rows)
        want = []
        for i, p in enumerate(pops):
            ranked = sorted([(err[k], cx[k], j) for k, (ii, j) in enumerate(pending)
                             if ii == i and hc[k]])
            want += [(i, j) for _, _, j in ranked[: H.admission_count(p, rows)]]
        assert got == sorted(want)
