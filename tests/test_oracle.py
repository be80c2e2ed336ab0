"""The CPU oracle, pinned against the golden fixtures and the reference's own
code; no GPU needed."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

CASES = sorted(d for d in os.listdir(GOLDEN) if os.path.isdir(os.path.join(GOLDEN, d)))


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("method", ["naive", "m4rm"])
def test_oracle_matches_golden(oracle, case, method):
    d = os.path.join(GOLDEN, case)
    expected = oracle.parse_answer(open(os.path.join(d, "expected.txt")).read())
    with oracle.Problem(os.path.join(d, "grammar.txt"), os.path.join(d, "graph.txt")) as p:
        p.closure(oracle.NAIVE if method == "naive" else oracle.M4RM, 2)
        assert p.results() == expected


def test_golden_has_every_kind():
    kinds = {c.split("_")[0] for c in CASES}
    assert {"known", "m4ricpu"} <= kinds


@pytest.mark.parametrize("case", [c for c in CASES if c.startswith("known")])
def test_reference_cpu_executable_on_known_answers(oracle, case):
    """The reference's own CPU main (built from its sources) reproduces the
    closed-form answers -- this pins the known-answer fixtures to the
    reference's driver and printer."""
    exe = oracle.ref_executable("m4riCPU")
    if exe is None:
        pytest.skip("oracle/_ref/m4riCPU not built")
    d = os.path.join(GOLDEN, case)
    got, _ = oracle.run_executable(exe, os.path.join(d, "grammar.txt"), os.path.join(d, "graph.txt"))
    assert got == oracle.parse_answer(open(os.path.join(d, "expected.txt")).read())


def _rows(rng, n, density):
    wpr = (n + 63) // 64
    bits = rng.random((n, wpr * 64)) < density
    bits[:, n:] = False
    return np.packbits(bits, axis=1, bitorder="little").view(np.uint64).reshape(n, wpr).copy()


def _dense(rows, n):
    return np.unpackbits(rows.view(np.uint8), axis=1, bitorder="little")[:, :n].astype(bool)


@pytest.mark.parametrize("n", [1, 5, 64, 65, 200, 333])
def test_products_agree_with_dense_definition(oracle, n):
    rng = np.random.default_rng(n)
    for density in (0.01, 0.1, 0.5):
        a, b, c = _rows(rng, n, density), _rows(rng, n, density), _rows(rng, n, density)
        exp = _dense(c, n) | (_dense(a, n).astype(np.int64) @ _dense(b, n).astype(np.int64) > 0)
        for method in (oracle.NAIVE, oracle.M4RM):
            cc = c.copy()
            changed = oracle.add_mul(cc, a, b, n, method, 2)
            assert np.array_equal(_dense(cc, n), exp)
            assert changed == (not np.array_equal(exp, _dense(c, n)))


def test_add_mul_aliasing_uses_old_values(oracle):
    n = 70
    rng = np.random.default_rng(1)
    c = _rows(rng, n, 0.05)
    d = _dense(c, n)
    exp = d | ((d.astype(np.int64) @ d.astype(np.int64)) > 0)
    cc = c.copy()
    oracle.add_mul(cc, cc, cc, n)  # the oracle's C code reads the snapshot
    assert np.array_equal(_dense(cc, n), exp)


def test_hash_count_is_the_reference_loop(oracle):
    rng = np.random.default_rng(7)
    for n in (1, 3, 64, 100):
        rows = _rows(rng, n, 0.3)
        bits = _dense(rows, n)
        h, count = 0, 0
        for r in range(n):
            line = 0
            for c in range(n):
                line = (line * 11 + int(bits[r, c])) % 1000000007
                count += int(bits[r, c])
            h = (h * 13 + line) % 1000000007
        assert oracle.hash_count(rows, n) == (h, count)


def test_grammar_parser_semantics(oracle, tmp_path):
    """First-seen numbering, arity dispatch, >3 tokens only registers the head,
    blank lines skipped (Grammar.cpp:17-51)."""
    g = tmp_path / "g.txt"
    g.write_text("S A B\n\nB b\nX y z w\nA a\nE\n")
    r = tmp_path / "r.txt"
    r.write_text("0 a 1\n1 b 2\n2 q 3\n")
    with oracle.Problem(str(g), str(r)) as p:
        assert p.names == ["S", "A", "B", "X", "E"]
        assert p.rules == [(0, 1, 2)]
        assert p.n == 4
        p.closure(oracle.NAIVE, 1)
        res = p.results()
    assert list(res) == ["A", "B", "E", "S", "X"]
    assert res["S"][1] == 1 and res["E"][1] == 4 and res["X"][1] == 0


def test_graph_loader_stops_at_malformed_line(oracle, tmp_path):
    g = tmp_path / "g.txt"
    g.write_text("S a\n")
    r = tmp_path / "r.txt"
    r.write_text("0 a 5\n1 a 2\nbroken line\n9 a 9\n")
    with oracle.Problem(str(g), str(r)) as p:
        assert p.n == 6
        p.closure(oracle.NAIVE, 1)
        assert p.results()["S"][1] == 2


def test_empty_graph(oracle, tmp_path):
    g = tmp_path / "g.txt"
    g.write_text("S A B\nA a\nB b\n")
    r = tmp_path / "r.txt"
    r.write_text("")
    with oracle.Problem(str(g), str(r)) as p:
        assert p.n == 0
        p.closure(oracle.M4RM, 1)
        assert p.results() == {"S": (0, 0), "A": (0, 0), "B": (0, 0)}


def test_hash_nibble_table_decomposition(oracle):
    """The decomposition the device hash uses equals the reference loop (the
    oracle): under a vertex order perm, with pow11[perm[c]] = 11^(n-1-c) and
    pow13[perm[r]] = 13^(n-1-r), a tile word's column term is the sum over
    its 16 nibbles of sub[tj][p][nibble] (the subset sums of the 4 column
    powers of nibble p), a row's terms add up over its tiles and are
    multiplied once by the row power."""
    p = 1000000007
    rng = np.random.default_rng(11)
    for n in (1, 63, 64, 130, 300):
        rows = _rows(rng, n, 0.2)
        bits = _dense(rows, n)
        perm = rng.permutation(n)
        T = (n + 63) // 64
        pow11 = np.zeros(T * 64, dtype=np.int64)
        pow13 = np.zeros(T * 64, dtype=np.int64)
        a = b = 1
        for c in range(n - 1, -1, -1):
            pow11[perm[c]], pow13[perm[c]] = a, b
            a, b = a * 11 % p, b * 13 % p
        sub = np.zeros((T, 16, 16), dtype=np.int64)
        for v in range(16):
            for bit in range(4):
                if (v >> bit) & 1:
                    sub[:, :, v] += pow11.reshape(T, 16, 4)[:, :, bit]
        sub %= p
        internal = np.zeros((T * 64, T * 64), dtype=bool)  # bit (perm[r], perm[c]) for vertex pair (r, c)
        rr, cc = np.nonzero(bits)
        internal[perm[rr], perm[cc]] = True
        h = 0
        for ti in range(T):
            for lane in range(64):
                acc = 0
                for tj in range(T):
                    word = 0
                    for k in np.nonzero(internal[ti * 64 + lane, tj * 64:(tj + 1) * 64])[0]:
                        word |= 1 << int(k)
                    acc += sum(int(sub[tj, q, (word >> (4 * q)) & 15]) for q in range(16))
                h += (acc % p) * int(pow13[ti * 64 + lane]) % p
        assert (h % p, int(bits.sum())) == oracle.hash_count(rows, n)
