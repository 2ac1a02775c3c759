"""The CPU restatement of the flat postfix variation engine (the checker of
the device's rc_pool_vary), pinned to the reference's own tests:
my-version/src/genome.rs:304-415 (width, Philox4x32-10 known answer,
position determinism) and my-version/src/postfix.rs:978-1209 (malformed
programs, bounded and valid children, the same position gives the same
child, islands independent of how many are evolved, front parents on and
off, dedup). Runs on the CPU."""
import importlib

import numpy as np

HALT = 255


def _pkg():
    return importlib.import_module("the-rule-and-compass_b200")


def _arena(O, islands, pop, seed, depth, err_fn):
    pkg = _pkg()
    w = O.random_arena(64, 2, 30, pkg.DEFAULT_VARIATION_OPS, seed, depth, islands * pop)
    err = np.array([err_fn(i) for i in range(islands * pop)], np.float64)
    return w, err


def test_width_and_philox_known_answer(O):
    pkg = _pkg()
    assert pkg.width_for(30) == 64 and pkg.width_for(0) == 8
    out = O.philox(0, 0, 0, 0)[0]
    assert [int(x) for x in out] == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]


def test_philox_is_position_determined(O):
    a = O.philox(9, 3, 7, 11)[0]
    assert np.array_equal(a, O.philox(9, 3, 7, 11)[0])
    for other in (O.philox(9, 4, 7, 11), O.philox(9, 3, 8, 11), O.philox(9, 3, 7, 12)):
        assert not np.array_equal(a, other[0])
    two = O.philox(9, 3, 7, 11, n=2)
    assert not np.array_equal(two[0], two[1])
    # the draw index (counter word 2) selects an attempt's stream
    assert not np.array_equal(a, O.philox(9, 3, 7, 11, draw=1)[0])


def test_spans_reject_malformed_programs(O):
    assert O.spans_count([2, HALT]) == -1
    assert O.spans_count([1, 0, HALT]) == 1
    assert O.spans_count([HALT]) == -1
    assert O.spans_count([1, 0, 1, 1, 2, HALT]) == 3


def test_variation_is_bounded_and_valid(O):
    pkg = _pkg()
    w, err = _arena(O, 3, 32, 7, 4, lambda i: abs(np.sin(i * 0.5)))
    words, ln, cost, h, e = O.next_generation(w, err, 3, 32, 64, 2, 30, 7, 1,
                                              pkg.DEFAULT_VARIATION_OPS)
    for k in range(3 * 32):
        assert ln[k] <= 64
        assert O.spans_count(words[k][:ln[k]]) == cost[k] >= 1
        assert cost[k] <= 30
        assert O.postfix_hash(words[k]) == h[k]


def test_the_same_position_gives_the_same_child(O):
    pkg = _pkg()
    w, err = _arena(O, 4, 40, 9, 3, lambda i: ((i * 37) % 101) / 101.0)
    a = O.next_generation(w, err, 4, 40, 64, 2, 30, 9, 3, pkg.DEFAULT_VARIATION_OPS)
    b = O.next_generation(w, err, 4, 40, 64, 2, 30, 9, 3, pkg.DEFAULT_VARIATION_OPS)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[3], b[3])
    assert np.array_equal(a[4].view(np.uint64), b[4].view(np.uint64))


def test_islands_do_not_depend_on_how_many_are_evolved(O):
    pkg = _pkg()
    w, err = _arena(O, 4, 24, 4, 3, lambda i: ((i * 13) % 97) / 97.0)
    four = O.next_generation(w, err, 4, 24, 64, 2, 30, 4, 2, pkg.DEFAULT_VARIATION_OPS)
    solo = O.next_generation(w[:24], err[:24], 1, 24, 64, 2, 30, 4, 2, pkg.DEFAULT_VARIATION_OPS)
    assert np.array_equal(four[0][:24], solo[0])
    assert np.array_equal(four[4][:24].view(np.uint64), solo[4].view(np.uint64))


def test_elite_survives_and_dedup_keeps_children_unique(O):
    pkg = _pkg()
    w, err = _arena(O, 2, 64, 9, 3, lambda i: ((i * 37) % 101) / 101.0)
    words, ln, cost, h, e = O.next_generation(w, err, 2, 64, 64, 2, 30, 9, 5,
                                              pkg.DEFAULT_VARIATION_OPS)
    parent_h = {O.postfix_hash(r) for r in w}
    for i in range(2):
        best = int(np.argmin(err[i * 64:(i + 1) * 64])) + i * 64
        assert np.array_equal(words[i * 64], w[best]) and e[i * 64] == err[best]
        assert np.all(np.isnan(e[i * 64 + 1:(i + 1) * 64]))
    kids = [int(x) for i in range(2) for x in h[i * 64 + 1:(i + 1) * 64]]
    assert len(set(kids)) == len(kids)
    assert not (set(kids) & parent_h)


def test_front_parents_change_children_and_the_off_path_is_unchanged(O):
    pkg = _pkg()
    w, err = _arena(O, 2, 64, 9, 3, lambda i: ((i * 37) % 101) / 101.0)
    front = [[1, 0, 0, np.float32(7.0).view(np.uint32), 2, HALT]]
    a = O.next_generation(w, err, 2, 64, 64, 2, 30, 9, 5, pkg.DEFAULT_VARIATION_OPS, front=front,
                          front_p=0.15)
    b = O.next_generation(w, err, 2, 64, 64, 2, 30, 9, 5, pkg.DEFAULT_VARIATION_OPS, front=front,
                          front_p=0.15)
    assert np.array_equal(a[0], b[0])
    off = O.next_generation(w, err, 2, 64, 64, 2, 30, 9, 5, pkg.DEFAULT_VARIATION_OPS)
    off2 = O.next_generation(w, err, 2, 64, 64, 2, 30, 9, 5, pkg.DEFAULT_VARIATION_OPS,
                             front=front, front_p=0.0)
    assert np.array_equal(off[0], off2[0])
    assert not np.array_equal(a[0], off[0])


def test_restart_replaces_the_island(O):
    pkg = _pkg()
    w, err = _arena(O, 2, 16, 3, 3, lambda i: float(i))
    words, ln, cost, h, e = O.next_generation(w, err, 2, 16, 64, 2, 30, 3, 4,
                                              pkg.DEFAULT_VARIATION_OPS, restart=[0, 1])
    assert np.all(np.isnan(e[16:]))
    for k in range(16, 32):
        assert O.spans_count(words[k][:ln[k]]) == cost[k] <= 30
