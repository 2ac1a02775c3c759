"""The device variation (rc_pool_vary) against the CPU restatement of the
reference engine (my-version/src/postfix.rs:511-973, genome.rs:43-302),
bit for bit: child programs, lengths, node counts, hashes and errors."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HALT = 255


def _evaluator(pkg):
    x = np.linspace(-1, 1, 64, dtype=np.float32)
    return pkg.GpuEvaluator(np.stack([x, x * x]).reshape(-1), 64, 2, x)


def _parents(pkg, O, islands, pop, width, nvars, mc, seed, depth, err_fn):
    w = O.random_arena(width, nvars, mc, pkg.DEFAULT_VARIATION_OPS, seed, depth, islands * pop)
    err = np.array([err_fn(i) for i in range(islands * pop)], np.float64)
    return w, err


def _same(dev, ref):
    dw, dl, dc, dh, de, ms = dev
    rw, rl, rc, rh, re = ref
    assert ms >= 0
    assert np.array_equal(dw, rw), np.argwhere(np.any(dw != rw, axis=1))[:5]
    assert np.array_equal(dl, rl) and np.array_equal(dc, rc)
    assert np.array_equal(dh, rh)
    assert np.array_equal(de.view(np.uint64), re.view(np.uint64))


def _case(pkg, O, islands, pop, width, nvars, mc, seed, gen, depth=3, err_fn=None, **kw):
    err_fn = err_fn or (lambda i: ((i * 37) % 101) / 101.0)
    w, err = _parents(pkg, O, islands, pop, width, nvars, mc, seed, depth, err_fn)
    ev = _evaluator(pkg)
    pool = pkg.GenomePool(ev, islands, pop, width)
    pool.upload(0, w)
    dev = pool.vary(0, err, gen, nvars, mc, seed, pkg.DEFAULT_VARIATION_OPS, **kw)
    ref = O.next_generation(w, err, islands, pop, width, nvars, mc, seed, gen,
                            pkg.DEFAULT_VARIATION_OPS, **kw)
    _same(dev, ref)
    assert np.array_equal(pool.hash(1), ref[3])
    ev.close()
    return dev, ref


def test_reference_configuration(pkg, O):
    _case(pkg, O, 3, 32, 64, 2, 30, 7, 1, depth=4, err_fn=lambda i: abs(np.sin(i * 0.5)))


def test_restart_island(pkg, O):
    _case(pkg, O, 4, 40, 64, 2, 30, 9, 3, restart=[0, 1, 0, 0])


def test_front_parents(pkg, O):
    front = [[1, 0, 0, int(np.float32(7.0).view(np.uint32)), 2, HALT],
             [1, 1, 9, HALT]]
    _case(pkg, O, 2, 64, 64, 2, 30, 9, 5, front=front, front_p=0.15)


def test_without_dedup(pkg, O):
    _case(pkg, O, 2, 48, 64, 3, 30, 11, 2, dedup=False)


def test_duplicate_heavy_population(pkg, O):
    """Tiny programs (at most 3 nodes, one input): most first attempts repeat
    a parent or an earlier child, so later attempts (computed on the host)
    and the random fallback after 64 attempts decide many slots."""
    _case(pkg, O, 4, 128, 10, 1, 3, 5, 7, depth=2)


def test_two_generations_ping_pong(pkg, O):
    islands, pop, width = 3, 48, 64
    w, err = _parents(pkg, O, islands, pop, width, 2, 30, 13, 3, lambda i: (i % 17) / 17.0)
    ev = _evaluator(pkg)
    pool = pkg.GenomePool(ev, islands, pop, width)
    pool.upload(0, w)
    d1 = pool.vary(0, err, 1, 2, 30, 13, pkg.DEFAULT_VARIATION_OPS)
    r1 = O.next_generation(w, err, islands, pop, width, 2, 30, 13, 1, pkg.DEFAULT_VARIATION_OPS)
    _same(d1, r1)
    err2 = np.array([(int(h) % 1000) / 1000.0 for h in r1[3]])
    d2 = pool.vary(1, err2, 2, 2, 30, 13, pkg.DEFAULT_VARIATION_OPS)
    r2 = O.next_generation(r1[0], err2, islands, pop, width, 2, 30, 13, 2,
                           pkg.DEFAULT_VARIATION_OPS)
    _same(d2, r2)
    ev.close()


def test_benchmark_sized_generation(pkg, O):
    """One generation of 16 islands x 1000 (the heavy-tailed configuration's
    population), width 64."""
    _case(pkg, O, 16, 1000, 64, 10, 30, 2024, 1, err_fn=lambda i: ((i * 7919) % 10007) / 10007.0)


def test_a_parent_that_is_not_a_program_fails_the_call(pkg, O):
    """A pool slot that is not a valid program (here an operator with no
    operands) fails the whole call: nothing is built from it, and the pool
    still serves the next, valid call."""
    islands, pop, width = 2, 50, 24
    w, err = _parents(pkg, O, islands, pop, width, 2, 10, 4, 3, lambda i: float(i))
    bad = w.copy()
    bad[17, :] = HALT
    bad[17, 0] = 2  # ADD with an empty stack
    ev = _evaluator(pkg)
    pool = pkg.GenomePool(ev, islands, pop, width)
    pool.upload(0, bad)
    with pytest.raises(pkg.DeviceError):
        pool.vary(0, err, 1, 2, 10, 4, pkg.DEFAULT_VARIATION_OPS)
    pool.upload(0, w)
    dev = pool.vary(0, err, 1, 2, 10, 4, pkg.DEFAULT_VARIATION_OPS)
    ref = O.next_generation(w, err, islands, pop, width, 2, 10, 4, 1, pkg.DEFAULT_VARIATION_OPS)
    _same(dev, ref)
    ev.close()
