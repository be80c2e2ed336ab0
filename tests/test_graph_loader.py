"""cfpq_graph_load, the parallel graph-file loader, against a literal
restatement of the reference's loop (cfpq-cpp/Graph.cpp:15,
`while (in >> from >> label >> to)`): whitespace tokens in triples, the list
ends at the first triple whose vertex tokens are not decimal numbers that fit
an unsigned int, n = max id + 1, labels numbered by first appearance.  No GPU
needed."""
import numpy as np
import pytest


def reference_parse(text: str):
    toks = text.split()
    src, lab, dst, lid = [], [], [], {}
    for i in range(0, len(toks) - 2, 3):
        a, l, b = toks[i:i + 3]
        if not (a.isdigit() and b.isdigit()) or int(a) > 0xFFFFFFFF or int(b) > 0xFFFFFFFF:
            break
        src.append(int(a))
        dst.append(int(b))
        lab.append(lid.setdefault(l, len(lid)))
    labels = sorted(lid, key=lid.get)
    n = max(src + dst) + 1 if src else 0
    return src, lab, dst, labels, n


def check(pkg, tmp_path, text, threads=(0, 1, 3, 7)):
    p = tmp_path / "g.txt"
    p.write_bytes(text.encode())
    exp = reference_parse(text)
    for t in threads:
        src, lab, dst, labels, n = pkg.capi.load_graph_file(str(p), t)
        assert src.tolist() == exp[0] and lab.tolist() == exp[1] and dst.tolist() == exp[2], t
        assert labels == exp[3] and n == exp[4], t
    return exp


def big_text(rng, m, nlab=5, n=10000):
    s, d, l = rng.integers(0, n, m), rng.integers(0, n, m), rng.integers(0, nlab, m)
    return "".join(f"{a} lab{c} {b}\n" for a, b, c in zip(s.tolist(), d.tolist(), l.tolist()))


def test_plain_and_whitespace_variants(pkg, tmp_path):
    rng = np.random.default_rng(1)
    text = big_text(rng, 200000)
    check(pkg, tmp_path, text)
    check(pkg, tmp_path, text.replace("\n", "\r\n"))              # CRLF
    check(pkg, tmp_path, text.replace(" ", "\t  "))              # tabs, runs of spaces
    check(pkg, tmp_path, "\n\n" + text.replace("\n", "\n\n", 500))  # blank lines
    check(pkg, tmp_path, text.rstrip("\n"))                      # no final newline
    check(pkg, tmp_path, "")
    check(pkg, tmp_path, "   \n\n")


def test_malformed_triple_ends_the_list(pkg, tmp_path):
    rng = np.random.default_rng(2)
    head, tail = big_text(rng, 120000), big_text(rng, 120000)
    for bad in ("x a 3\n", "1 a -2\n", "4294967296 a 1\n", "12abc a 3\n", "1 a 2.0\n"):
        exp = check(pkg, tmp_path, head + bad + tail)
        assert len(exp[0]) == 120000
    check(pkg, tmp_path, head + "4294967294 a 0\n" + tail)  # the largest id whose count fits


def test_triples_across_lines_fall_back_to_the_token_stream(pkg, tmp_path):
    rng = np.random.default_rng(3)
    text = big_text(rng, 150000)
    words = text.split()
    odd = "\n".join(" ".join(words[i:i + 2]) for i in range(0, len(words), 2)) + "\n"  # 2 tokens per line
    exp = check(pkg, tmp_path, odd)
    assert len(exp[0]) == 150000
    check(pkg, tmp_path, "1 a\n2 3 b 4\n5 c 6\n")


def test_many_labels_numbered_by_first_appearance(pkg, tmp_path):
    lines = [f"{i} l{(i * 7919) % 3001} {i + 1}\n" for i in range(100000)]
    check(pkg, tmp_path, "".join(lines))


def test_edge_graph_and_errors(pkg, tmp_path):
    p = tmp_path / "g.txt"
    p.write_text("0 a 1\n1 b 2\n")
    g = pkg.query.EdgeGraph.from_file(str(p))
    assert g.n == 3 and g.labels == ["a", "b"] and g.nedges == 2
    with pytest.raises(pkg.capi.CfpqError) as e:
        pkg.capi.load_graph_file(str(tmp_path / "missing.txt"))
    assert e.value.code == pkg.capi.ERR_IO
