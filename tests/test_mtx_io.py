"""MatrixMarket / binary matrix I/O (host code behind the C ABI) against the
reference's own known answers (tests/golden/mtx_cases.json, extracted from
core/test/base/mtx_io.cpp) and against the oracle's restatement of
core/base/mtx_io.cpp on seeded generated files."""
import base64
import json
import os

import numpy as np
import pytest

from ginkgo_b200 import mtx_io as M
from ginkgo_b200._lib import GinkgoError
from oracle import mtx as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
with open(os.path.join(ROOT, "tests", "golden", "mtx_cases.json")) as f:
    CASES = json.load(f)

NP_VT = {"f64": np.float64, "f32": np.float32}
NP_IT = {"i32": np.int32, "i64": np.int64}


def _rounded(entries, vt):
    return [(int(r), int(c), float(NP_VT[vt](v))) for r, c, v in entries]


def _lib_read(src, reader, vt, it):
    fn = {"raw": M.read_raw, "generic_raw": M.read_generic_raw,
          "binary_raw": M.read_binary_raw}[reader]
    return fn(src, NP_VT[vt], NP_IT[it])


def _oracle_read(src, reader, vt, it):
    if reader == "raw":
        return O.read_raw(src, vt, it)
    if reader == "generic_raw":
        return O.read_generic_raw(src if isinstance(src, bytes) else src.encode(), vt, it)
    return O.read_binary_raw(src, vt, it)


def _read_cases():
    for c in CASES["read"]:
        yield c, c["text"]
    for c in CASES["binary_read"]:
        yield c, base64.b64decode(c["bytes"])


READS = list(_read_cases())


@pytest.mark.parametrize("case,src", READS,
                         ids=[f"{c['name']}-{c['value_type']}-{c['index_type']}" for c, _ in READS])
def test_reads_match_reference_known_answers(case, src):
    vt, it = case["value_type"], case["index_type"]
    if case.get("error"):
        with pytest.raises(GinkgoError):
            _lib_read(src, case["reader"], vt, it)
        with pytest.raises(O.MtxError):
            _oracle_read(src, case["reader"], vt, it)
        return
    expected = _rounded(case["entries"], vt)
    d = _lib_read(src, case["reader"], vt, it)
    assert d.size == tuple(case["size"])
    assert d.values.dtype == NP_VT[vt] and d.row_idxs.dtype == NP_IT[it]
    assert d.nonzeros == expected
    size, entries = _oracle_read(src, case["reader"], vt, it)
    assert size == tuple(case["size"]) and entries == expected


@pytest.mark.parametrize("case", CASES["write"], ids=[c["name"] for c in CASES["write"]])
def test_writes_match_reference_known_answers(case):
    vt = NP_VT[case["value_type"]]
    entries = [(i, j, v) for i, row in enumerate(case["dense"])
               for j, v in enumerate(row) if v != 0]
    size = (len(case["dense"]), max(len(r) for r in case["dense"]))
    data = M.MatrixData.from_entries(size, entries, vt, NP_IT[case["index_type"]])
    assert M.write_raw(data, case["layout"]) == case["expected"]
    assert O.write_raw(size, _rounded(entries, case["value_type"]), case["layout"]) == \
        case["expected"]


def test_binary_write_matches_reference_known_answer():
    case = CASES["binary_write"][0]
    expected = base64.b64decode(case["expected"])
    data = M.MatrixData.from_entries(case["size"], case["entries"], NP_VT[case["value_type"]],
                                     NP_IT[case["index_type"]])
    assert M.write_binary_raw(data) == expected
    assert O.write_binary_raw(tuple(case["size"]), case["entries"], case["value_type"],
                              case["index_type"]) == expected


# --------------------------------------------------------------- generated --

def _fmt_value(rng, v, field):
    if field == "integer":
        return str(int(v))
    k = rng.integers(6)
    if k == 0:
        return repr(float(v))
    if k == 1:
        return "%.17g" % v
    if k == 2:
        return "%e" % v
    if k == 3:
        return "%E" % v
    if k == 4:
        return ("+" if v >= 0 else "") + "%.9g" % v
    s = "%.6f" % v  # leading-dot form where it applies
    return s.replace("0.", ".", 1) if s.startswith("0.") else s


def _gen_mtx(rng):
    layout = ["coordinate", "array"][rng.integers(2)]
    field = ["real", "integer", "pattern"][rng.integers(3)]
    modifier = ["general", "symmetric", "skew-symmetric", "hermitian"][rng.integers(4)]
    n = int(rng.integers(1, 9))
    m = n if modifier != "general" else int(rng.integers(1, 9))
    nl = "\r\n" if rng.integers(4) == 0 else "\n"
    head = "%%MatrixMarket matrix {} {} {}".format(layout, field, modifier)
    if rng.integers(2):
        head = "".join(ch.upper() if rng.integers(2) else ch for ch in head)
    if rng.integers(3) == 0:
        head += " trailing words"
    lines = [""] * int(rng.integers(2)) + [head]
    lines += ["% comment " + str(i) for i in range(int(rng.integers(3)))]

    def val():
        v = rng.normal() * 10.0 ** int(rng.integers(-3, 4))
        return float(np.round(v)) if field == "integer" else float(v)

    def junk():
        return ["", "", " x y", "\t% tail", " 7"][rng.integers(5)]

    sep = lambda: [" ", "  ", "\t"][rng.integers(3)]  # noqa: E731
    if layout == "coordinate":
        pos = []
        for i in range(n):
            for j in range(m):
                lower = j <= i if modifier != "skew-symmetric" else j < i
                if (modifier == "general" or lower) and rng.random() < 0.5:
                    pos.append((i, j))
        rng.shuffle(pos)
        lines.append(f"{n}{sep()}{m}{sep()}{len(pos)}" + junk())
        for i, j in pos:
            s = f"{i + 1}{sep()}{j + 1}"
            if field != "pattern":
                s += sep() + _fmt_value(rng, val(), field)
            lines.append(s + junk())
    else:
        lines.append(f"{n}{sep()}{m}" + junk())
        for j in range(m):
            r0 = {"general": 0, "skew-symmetric": j + 1}.get(modifier, j)
            for i in range(r0, n):
                lines.append((_fmt_value(rng, val(), field) if field != "pattern" else "")
                             + junk())
    return nl.join(lines) + nl


@pytest.mark.parametrize("seed", range(40))
def test_reads_match_oracle_on_generated_files(seed):
    rng = np.random.default_rng(seed)
    for _ in range(10):
        text = _gen_mtx(rng)
        for vt in ("f64", "f32"):
            for it in ("i32", "i64"):
                try:
                    size, entries = O.read_raw(text, vt, it)
                except O.MtxError:
                    # e.g. a blank first line with CRLF endings is "\r",
                    # not empty, and fails as a header in the reference too
                    with pytest.raises(GinkgoError):
                        M.read_raw(text, NP_VT[vt], NP_IT[it])
                    continue
                d = M.read_raw(text, NP_VT[vt], NP_IT[it])
                assert d.size == size, text
                assert d.nonzeros == entries, text
                # generic: text only when the first byte is '%' (a leading
                # blank line sends it to the binary reader, as in the reference)
                raw = text.encode()
                if raw[:1] == b"%":
                    g = M.read_generic_raw(raw, NP_VT[vt], NP_IT[it])
                    assert g.nonzeros == O.read_generic_raw(raw, vt, it)[1] == entries
                else:
                    with pytest.raises(O.MtxError):
                        O.read_generic_raw(raw, vt, it)
                    with pytest.raises(GinkgoError):
                        M.read_generic_raw(raw, NP_VT[vt], NP_IT[it])


@pytest.mark.parametrize("seed", range(10))
def test_write_read_round_trips(seed):
    rng = np.random.default_rng(100 + seed)
    n, m = int(rng.integers(1, 30)), int(rng.integers(1, 30))
    k = int(rng.integers(0, n * m + 1))
    flat = rng.choice(n * m, size=k, replace=False)
    entries = sorted((int(f // m), int(f % m), float(rng.normal())) for f in flat)
    for vt, it in (("f64", "i32"), ("f32", "i64")):
        data = M.MatrixData.from_entries((n, m), entries, NP_VT[vt], NP_IT[it])
        ent = _rounded(entries, vt)
        # binary: exact both ways
        b = M.write_binary_raw(data)
        assert b == O.write_binary_raw((n, m), ent, vt, it)
        assert M.read_binary_raw(b, NP_VT[vt], NP_IT[it]).nonzeros == ent
        # text: six significant digits, as the reference's stream writes them
        for layout in ("coordinate", "array"):
            t = M.write_raw(data, layout)
            assert t == O.write_raw((n, m), ent, layout)
            back = M.read_raw(t, NP_VT[vt], NP_IT[it])
            assert back.nonzeros == O.read_raw(t, vt, it)[1]
            if layout == "coordinate":
                assert [(r, c) for r, c, _ in back.nonzeros] == [(r, c) for r, c, _ in ent]
                np.testing.assert_allclose(back.values, [v for _, _, v in ent], rtol=1e-5)


BAD_TEXT = [
    "",
    "\n\n",
    "%%MatrixMarket matrix coordinate real\n1 1 1\n1 1 1.0\n",
    "%%MatrixMarket tensor coordinate real general\n1 1 1\n1 1 1.0\n",
    "%%MatrixMarket matrix coordinate real general\n",
    "%%MatrixMarket matrix coordinate real general\n% only comments\n",
    "%%MatrixMarket matrix coordinate real general\n\n1 1 1\n1 1 1.0\n",
    "%%MatrixMarket matrix coordinate real general\n2 2\n1 1 1.0\n",
    "%%MatrixMarket matrix coordinate real general\n-2 2 1\n1 1 1.0\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1.0\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n1 x 1.0\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 abc\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 1e\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 .\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n3000000000 1 1.0\n",
    "%%MatrixMarket matrix coordinate complex general\n2 2 1\n1 1 1.0 2.0\n",
    "%%MatrixMarket matrix array real general\n2 2\n1.0\n2.0\n3.0\n",
    "%%MatrixMarket matrix array real general\n2\n1.0\n",
]


@pytest.mark.parametrize("text", BAD_TEXT)
def test_malformed_text_fails_in_both(text):
    with pytest.raises(O.MtxError):
        O.read_raw(text, "f64", "i32")
    with pytest.raises(GinkgoError):
        M.read_raw(text)


def test_int64_indices_take_what_int32_rejects():
    text = "%%MatrixMarket matrix coordinate real general\n2 2 1\n3000000000 1 1.0\n"
    d = M.read_raw(text, np.float64, np.int64)
    assert d.nonzeros == O.read_raw(text, "f64", "i64")[1] == [(2999999999, 0, 1.0)]


def test_malformed_binary_fails_in_both():
    good = M.write_binary_raw(M.MatrixData.from_entries((4, 4), [(0, 0, 1.0), (3, 2, 2.0)]))
    bad_magic = b"GINKGOQI" + good[8:]
    cases = [b"", good[:31], good[:-1], bad_magic]
    big = bytearray(good)
    big[8:16] = (2**33).to_bytes(8, "little")  # rows beyond int32
    for data in cases + [bytes(big)]:
        with pytest.raises(O.MtxError):
            O.read_binary_raw(data, "f64", "i32")
        with pytest.raises(GinkgoError):
            M.read_binary_raw(data)
    # the same oversized header is fine for int64 indices
    assert M.read_binary_raw(bytes(big), np.float64, np.int64).size == (2**33, 4)


def test_binary_half_and_bfloat16_files():
    vals = [1.0, -2.5, 65504.0, 2.0**-24, 0.0]
    n = len(vals)
    import struct
    for letter, pack in (("H", lambda v: struct.pack("<e", v)),
                         ("B", lambda v: struct.pack("<f", v)[2:])):
        data = b"GINKGO" + letter.encode() + b"I" + struct.pack("<3Q", n, n, n)
        data += b"".join(struct.pack("<ii", i, i) + pack(v) for i, v in enumerate(vals))
        for vt in ("f64", "f32"):
            exp = O.read_binary_raw(data, vt, "i32")[1]
            assert M.read_binary_raw(data, NP_VT[vt], np.int32).nonzeros == exp
    assert exp[0] == (0, 0, 1.0)


def test_csr_arrays_from_matrix_data():
    text = ("%%MatrixMarket matrix coordinate real symmetric\n4 4 5\n"
            "1 1 4\n2 1 -1\n2 2 4\n4 3 -1\n4 4 4\n")
    d = M.read_raw(text)
    rp, ci, v = M.data_to_csr_arrays(d)
    dense = np.zeros((4, 4))
    for r in range(4):
        for k in range(rp[r], rp[r + 1]):
            dense[r, ci[k]] += v[k]
    expected = np.array([[4, -1, 0, 0], [-1, 4, 0, 0], [0, 0, 0, -1], [0, 0, -1, 4.0]])
    assert np.array_equal(dense, expected)
    assert rp.dtype == np.int32 and ci.dtype == np.int32
    with pytest.raises(ValueError):
        M.data_to_csr_arrays(M.read_raw(
            "%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1.0\n"))


@pytest.mark.parametrize("value,ok", [
    ("1e400", False), ("-1e400", False), ("1.8e308", False), ("1.7e308", True),
    ("1e-400", True), ("4.9e-324", True), ("2.4e-324", True), ("-2.5e-324", True),
    ("+.5", True), ("5.", True), ("007", True), ("-0", True)])
def test_overflow_fails_and_underflow_rounds_like_the_stream(value, ok):
    text = f"%%MatrixMarket matrix coordinate real general\n1 1 1\n1 1 {value}\n"
    if not ok:
        with pytest.raises(O.MtxError):
            O.read_raw(text)
        with pytest.raises(GinkgoError):
            M.read_raw(text)
        return
    exp = O.read_raw(text)[1]
    got = M.read_raw(text).nonzeros
    assert got == exp and np.signbit(got[0][2]) == np.signbit(exp[0][2])
    # FP32 storage rounds the double (1.7e308 becomes inf there, as a cast does)
    assert M.read_raw(text, np.float32).nonzeros == O.read_raw(text, "f32")[1]


def _big_coordinate_text(rng, n, per_row, symmetric=False):
    """A coordinate file of about n * per_row entries (> 8 MB, so the reader
    takes its parallel path), rows shuffled."""
    rows, cols = [], []
    for k in range(per_row):
        r = np.arange(n)
        c = (r + k * 7919) % n if not symmetric else np.maximum(r - k, 0)
        rows.append(r)
        cols.append(c)
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    keep = np.ones(len(r), bool)
    if symmetric:  # unique lower-triangle positions
        key = r * n + c
        _, first = np.unique(key, return_index=True)
        keep[:] = False
        keep[first] = True
    r, c = r[keep], c[keep]
    perm = rng.permutation(len(r))
    r, c = r[perm], c[perm]
    v = rng.standard_normal(len(r)) * 10.0 ** rng.integers(-5, 6, len(r))
    body = "\n".join(f"{a + 1} {b + 1} {x!r}" for a, b, x in zip(r.tolist(), c.tolist(), v.tolist()))
    kind = "symmetric" if symmetric else "general"
    return f"%%MatrixMarket matrix coordinate real {kind}\n{n} {n} {len(r)}\n{body}\n"


@pytest.mark.parametrize("symmetric", [False, True])
def test_large_file_parallel_path_matches_oracle(symmetric):
    rng = np.random.default_rng(7 + symmetric)
    text = _big_coordinate_text(rng, 50_000, 9, symmetric)
    assert len(text) > 9 << 20
    size, entries = O.read_raw(text)
    d = M.read_raw(text)
    assert d.size == size
    assert np.array_equal(d.row_idxs, [e[0] for e in entries])
    assert np.array_equal(d.col_idxs, [e[1] for e in entries])
    assert np.array_equal(d.values, [e[2] for e in entries])


def test_large_file_irregular_lines_fall_back_to_the_stream_rules():
    rng = np.random.default_rng(11)
    base = _big_coordinate_text(rng, 40_000, 9)
    head, dims, body = base.split("\n", 2)
    lines = body.split("\n")
    nnz = int(dims.split()[2])
    mid = len(lines) // 2
    variants = {
        # the value of one entry on the next line: still valid for a stream
        "split": lines[:mid] + [" ".join(lines[mid].split()[:2]), lines[mid].split()[2]]
        + lines[mid + 1:],
        # blank lines between entries
        "blank": lines[:mid] + ["", "   \t"] + lines[mid:],
        # garbage after the last entry is never read
        "tail": lines[:nnz] + ["not an entry", "%"],
        # a comment line in the middle is an error
        "comment": lines[:mid] + ["% comment"] + lines[mid:],
        # one entry too few
        "short": lines[:nnz - 1],
    }
    for name, ls in variants.items():
        text = f"{head}\n{dims}\n" + "\n".join(ls) + "\n"
        try:
            size, entries = O.read_raw(text)
        except O.MtxError:
            with pytest.raises(GinkgoError):
                M.read_raw(text)
            assert name in ("comment", "short")
            continue
        assert name in ("split", "blank", "tail")
        d = M.read_raw(text)
        assert d.size == size
        assert np.array_equal(d.values, [e[2] for e in entries]), name
        assert np.array_equal(d.row_idxs, [e[0] for e in entries]), name
        assert np.array_equal(d.col_idxs, [e[1] for e in entries]), name


def test_large_write_matches_oracle_format():
    rng = np.random.default_rng(5)
    n = 300_000
    r = np.sort(rng.integers(0, 100_000, n)).astype(np.int32)
    c = rng.integers(0, 100_000, n).astype(np.int32)
    v = rng.standard_normal(n) * 10.0 ** rng.integers(-8, 9, n)
    data = M.MatrixData((100_000, 100_000), r, c, v)
    text = M.write_raw(data)
    ent = list(zip(r.tolist(), c.tolist(), v.tolist()))
    assert text == O.write_raw((100_000, 100_000), ent)


def test_dense_read_and_write_follow_dense_read_write():
    import torch
    text = ("%%MatrixMarket matrix coordinate real general\n3 2 4\n"
            "1 1 1.5\n3 2 -2\n1 1 7\n2 1 0.25\n")
    t = M.read_dense(text)
    size, entries = O.read_raw(text)
    exp = np.zeros(size)
    for r, c, v in entries:  # Dense::read assigns in order: the later 1 1 wins
        exp[r, c] = v
    assert t.dtype == torch.float64 and np.array_equal(t.numpy(), exp)
    assert M.read_dense(text, dtype=torch.float32).dtype == torch.float32
    # write: nonzeros row-major; array once a quarter is nonzero
    a = torch.zeros(8, 3, dtype=torch.float64)
    a[1, 2], a[5, 0] = 3.5, -1.0
    ent = [(1, 2, 3.5), (5, 0, -1.0)]
    assert M.write_dense(a) == O.write_raw((8, 3), ent, "coordinate")
    a[:3, :] = 1.0
    ent = [(i, j, float(a[i, j])) for i in range(8) for j in range(3) if a[i, j] != 0]
    assert M.write_dense(a) == O.write_raw((8, 3), ent, "array")
    assert np.array_equal(M.read_dense(M.write_dense(a)).numpy(), a.numpy())
