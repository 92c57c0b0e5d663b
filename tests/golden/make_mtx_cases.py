"""Writes tests/golden/mtx_cases.json: the known answers of the reference's
MatrixMarket / binary I/O tests (core/test/base/mtx_io.cpp of Ginkgo 1.12),
extracted from that test source as text.

Kept: every case on real value types (double, float) with int32/int64
indices — text reads with their expected size and entries, the reads that
must fail, the writer cases with their expected text, and the binary read /
write cases with their byte images.  Complex-valued cases are skipped (the
path is real-valued) except where a real read of complex data must fail.
Each case carries the file:line of its TEST.

Run:  python tests/golden/make_mtx_cases.py <path to the reference tree>
"""
import base64
import json
import os
import re
import struct
import sys

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_mtx_cases.py <path to the reference tree>")
REF = sys.argv[1]
SRC = os.path.join(REF, "core", "test", "base", "mtx_io.cpp")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mtx_cases.json")

text = open(SRC).read()

VT = {"double": "f64", "float": "f32"}
IT = {"gko::int32": "i32", "gko::int64": "i64", "int": "i32"}


def body_of(start):
    """The brace-balanced body after text offset start, and its end."""
    i = text.index("{", start)
    depth = 0
    for j in range(i, len(text)):
        if text[j] == "{":
            depth += 1
        elif text[j] == "}":
            depth -= 1
            if depth == 0:
                return text[i + 1:j], j
    raise ValueError("unbalanced braces")


def c_strings(s):
    """Concatenation of the C string literals in s."""
    out = []
    for lit in re.findall(r'"((?:[^"\\]|\\.)*)"', s):
        out.append(lit.encode().decode("unicode_escape"))
    return "".join(out)


def line_of(off):
    return text.count("\n", 0, off) + 1


def num(tok):
    tok = tok.strip()
    return float(tok) if any(ch in tok for ch in ".eE") else int(tok)


def binary_words(func):
    """Byte image of build_binary_<func>_data(): the uint64 initializer list;
    the magic is the character literals in order (least significant first),
    int_val / neg_int_val are the bits of the doubles declared above them."""
    m = re.search(r"build_binary_%s_data\(\)" % func, text)
    body, _ = body_of(m.end())
    dbl = dict(re.findall(r"double (\w+) = (-?[\d.]+);", body))
    alias = {a: float(dbl[b]) for a, b in
             re.findall(r"std::memcpy\(&(\w+), &(\w+), sizeof\(double\)\);", body)}
    init = body[body.index("data{") + 5:body.rindex("}")]
    init = re.sub(r"//[^\n]*", "", init)
    words = []
    depth, tok = 0, ""
    for ch in init:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == "," and depth == 0:
            words.append(tok.strip())
            tok = ""
        else:
            tok += ch
    if tok.strip():
        words.append(tok.strip())
    out = b""
    for w in words:
        if "'" in w:
            out += "".join(re.findall(r"'(.)'", w)).encode()
        elif w in alias:
            out += struct.pack("<d", alias[w])
        else:
            out += struct.pack("<Q", int(w))
    return out


cases = {"_about": __doc__.strip().splitlines()[0], "read": [], "write": [],
         "binary_read": [], "binary_write": []}

for m in re.finditer(r"^TEST\((MtxReader|MatrixData), (\w+)\)", text, flags=re.M):
    name = f"{m.group(1)}.{m.group(2)}"
    body, end = body_of(m.end())
    src = f"core/test/base/mtx_io.cpp:{line_of(m.start())}-{line_of(end)}"
    rd = re.search(r"gko::read_(raw|generic_raw)<([\w:]+), ([\w:]+)>\(iss\)", body)
    if "std::istringstream iss(" in body and rd:
        vt, it = rd.group(2), rd.group(3)
        if vt not in VT:
            continue
        lit = body[body.index("std::istringstream iss(") + 23:]
        lit = lit[:lit.index(");")]
        case = {"name": name, "source": src, "text": c_strings(lit),
                "reader": rd.group(1), "value_type": VT[vt], "index_type": IT[it]}
        if "ASSERT_THROW" in body:
            case["error"] = True
        else:
            sz = re.search(r"ASSERT_EQ\(data\.size, gko::dim<2>\((\d+), (\d+)\)\)", body)
            case["size"] = [int(sz.group(1)), int(sz.group(2))]
            case["entries"] = [[int(r), int(c), float(v)] for r, c, v in re.findall(
                r"ASSERT_EQ\(v\[\d+\], tpl\((-?\d+), (-?\d+), ([-\d.eE+]+)\)\)", body)]
        cases["read"].append(case)
    elif "write_raw(oss, data" in body:
        dm = re.search(r"gko::matrix_data<([\w:]+), ([\w:]+)> data\{(.*?)\};", body, flags=re.S)
        if dm is None or dm.group(1) not in VT:  # complex values
            continue
        vt, it = dm.group(1), dm.group(2)
        init = re.sub(r"//[^\n]*", "", dm.group(3))
        rows = [[num(t) for t in r.split(",")] for r in re.findall(r"\{([^{}]*)\}", init)]
        layout = "array" if "layout_type::array" in body else "coordinate"
        exp = body[body.index("ASSERT_EQ(oss.str(),") + 20:]
        exp = exp[:exp.index(");")]
        cases["write"].append({"name": name, "source": src, "value_type": VT[vt],
                               "index_type": IT[it], "dense": rows, "layout": layout,
                               "expected": c_strings(exp)})

# binary reads: the real and complex byte images and the expected entries
real_img, cplx_img = binary_words("real"), binary_words("complex")
for tname, img in (("ReadsBinary", real_img), ("ReadsComplexBinary", cplx_img)):
    m = re.search(r"^TEST\(MtxReader, %s\)" % tname, text, flags=re.M)
    body, end = body_of(m.end())
    src = f"core/test/base/mtx_io.cpp:{line_of(m.start())}-{line_of(end)}"
    body_nohalf = re.sub(r"#if GINKGO_ENABLE_\w+.*?#endif", "", body, flags=re.S)
    for fn, vt, it in re.findall(r"(test_read(?:_fail)?)\(gko::matrix_data<([\w:]+), ([\w:]+)>\{\}\)",
                                 body_nohalf):
        if vt not in VT:
            continue
        case = {"name": f"MtxReader.{tname}", "source": src, "value_type": VT[vt],
                "index_type": IT[it], "reader": "binary_raw",
                "bytes": base64.b64encode(img).decode()}
        if fn == "test_read_fail":
            case["error"] = True
        else:
            sz = re.search(r"ASSERT_EQ\(data\.size, gko::dim<2>\((\d+), (\d+)\)\)", body)
            get = lambda f: [num(x) for _, x in sorted(
                re.findall(r"ASSERT_EQ\(data\.nonzeros\[(\d)\]\.%s, ([^)]+)\);" % f, body))]
            vals = [float(re.sub(r"value_type\{(.*)\}", r"\1", v)) for _, v in sorted(
                re.findall(r"ASSERT_EQ\(data\.nonzeros\[(\d)\]\.value, (value_type\{[^}]*\})\);", body))]
            case["size"] = [int(sz.group(1)), int(sz.group(2))]
            case["entries"] = [[r, c, v] for r, c, v in zip(get("row"), get("column"), vals)]
        cases["binary_read"].append(case)

m = re.search(r"^TEST\(MtxReader, ReadsGenericBinary\)", text, flags=re.M)
body, end = body_of(m.end())
gm = re.search(r"read_generic_raw<(\w+), (\w+)>", body)
cases["binary_read"].append({
    "name": "MtxReader.ReadsGenericBinary",
    "source": f"core/test/base/mtx_io.cpp:{line_of(m.start())}-{line_of(end)}",
    "value_type": VT[gm.group(1)], "index_type": IT[gm.group(2)], "reader": "generic_raw",
    "bytes": base64.b64encode(real_img).decode(),
    "size": [int(x) for x in re.search(r"gko::dim<2>\((\d+), (\d+)\)", body).groups()],
    "entries": [[r, c, v] for r, c, v in zip(
        [int(x) for _, x in sorted(re.findall(r"nonzeros\[(\d)\]\.row, (\d+)\)", body))],
        [int(x) for _, x in sorted(re.findall(r"nonzeros\[(\d)\]\.column, (\d+)\)", body))],
        [float(x) for _, x in sorted(re.findall(r"nonzeros\[(\d)\]\.value, (-?[\d.]+)\)", body))])]})

m = re.search(r"^TEST\(MtxReader, WritesBinary\)", text, flags=re.M)
body, end = body_of(m.end())
dm = re.search(r"gko::matrix_data<([\w:]+), ([\w:]+)> data;", body)
cases["binary_write"].append({
    "name": "MtxReader.WritesBinary",
    "source": f"core/test/base/mtx_io.cpp:{line_of(m.start())}-{line_of(end)}",
    "value_type": VT[dm.group(1)], "index_type": IT[dm.group(2)],
    "size": [int(x) for x in re.search(r"gko::dim<2>\{(\d+), (\d+)\}", body).groups()],
    "entries": [[int(r), int(c), float(v)] for _, r, c, v in sorted(re.findall(
        r"data\.nonzeros\[(\d)\] = \{(-?\d+), (-?\d+), (-?[\d.]+)\};", body))],
    "expected": base64.b64encode(real_img).decode()})

with open(OUT, "w") as f:
    json.dump(cases, f, indent=1)
    f.write("\n")
print({k: len(v) for k, v in cases.items() if isinstance(v, list)})
