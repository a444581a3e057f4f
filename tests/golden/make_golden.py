"""Generate tests/golden/groupby_multikeys.json from the reference's own tests.

Reads the reference project's src/cuda/tests/groupby/groupby_multikeys_test.cu
as text and extracts, for every TEST_P case, its input arrays, which arrays
form the key and value tables, the aggregation requests, the hint flags, and
the expected results the test asserts (std::map `expected` literals, the
per-key if/else EXPECT blocks and single-row EXPECTs).  Nothing is executed.

Run with the path of a checkout of the reference project:
    python tests/golden/make_golden.py REF
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
REF = Path(sys.argv[1])
SRC = REF / "src/cuda/tests/groupby/groupby_multikeys_test.cu"
OUT = Path(__file__).resolve().parent / "groupby_multikeys.json"

CTYPE = {"int32_t": "int32", "int64_t": "int64", "float": "float32", "double": "float64"}


def split_top(s: str) -> list[str]:
    """Split a brace-list body on top-level commas."""
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch in "{(":
            depth += 1
        elif ch in "})":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur.strip())
    return out


def strip_braces(s: str) -> str:
    s = s.strip()
    if s.startswith("{") and s.endswith("}"):
        return s[1:-1]
    return s


def num(s: str):
    s = s.strip().rstrip("fF")
    return float(s) if any(c in s for c in ".eE") else int(s)


def brace_block(text: str, start: int) -> tuple[str, int]:
    """Return the {...} block starting at text[start] == '{' (exclusive) and end index."""
    assert text[start] == "{"
    depth = 0
    for i in range(start, len(text)):
        if text[i] == "{":
            depth += 1
        elif text[i] == "}":
            depth -= 1
            if depth == 0:
                return text[start + 1:i], i + 1
    raise ValueError("unbalanced braces")


def parse_case(name: str, body: str) -> dict:
    case = {"name": name, "ok": True, "notes": []}
    arrays = {}
    for m in re.finditer(r"\b(int32_t|int64_t|float|double)\s+(\w+)\[\]\s*=\s*\{([^}]*)\};", body):
        arrays[m.group(2)] = {"dtype": CTYPE[m.group(1)], "values": [num(x) for x in m.group(3).split(",") if x.strip()]}
    colvar = {m.group(1): m.group(2) for m in re.finditer(r"auto\s+(\w+)\s*=\s*gamax::make_column_from_host\((\w+),", body)}
    keys = [colvar.get(m.group(1)) for m in re.finditer(r"key_columns\.push_back\(std::move\((\w+)\)\)", body)]
    vals = [colvar.get(m.group(1)) for m in re.finditer(r"val_columns\.push_back\(std::move\((\w+)\)\)", body)]
    if not arrays or None in keys or None in vals or not keys:
        case["ok"] = False
        case["notes"].append("inputs are not literal arrays")
        return case
    case["keys"] = [arrays[k] for k in keys]
    case["vals"] = [arrays[v] for v in vals]
    case["requests"] = [[int(m.group(1)), m.group(2)] for m in
                        re.finditer(r"requests\.push_back\(\{(\d+),\s*gamax::groupby::aggregation_id::(\w+)\}\)", body)]
    case["agg_count"] = bool(re.search(r"hint\.agg_count\s*=\s*true", body))
    m = re.search(r"EXPECT_EQ\(result->num_rows\(\),\s*(\d+)\)", body)
    case["num_rows"] = int(m.group(1)) if m else None
    m = re.search(r"EXPECT_EQ\(result->num_columns\(\),\s*(\d+)\)", body)
    case["num_columns"] = int(m.group(1)) if m else None
    case["column_types"] = {m.group(1): m.group(2) for m in re.finditer(
        r"EXPECT_EQ\(result->get_column\((\d+)\)\.type\(\)\.id\(\),\s*gamax::type_id::(\w+)\)", body)}
    hcol = {m.group(1): int(m.group(2)) for m in re.finditer(
        r"auto\s+(h_\w+)\s*=\s*gamax::copy_column_to_host<\w+>\(result->get_column\((\d+)\)", body)}
    nkeys = len(keys)
    key_names = [n for n, c in hcol.items() if c < nkeys]
    key_names.sort(key=lambda n: hcol[n])
    expects = []  # {"key": [..] or "row": r, "column": c, "value": v, "tol": t}

    # Form 1: std::map<...> expected = { ... };
    m = re.search(r"std::map<.*?>\s+expected\s*=\s*", body)
    if m:
        blk, _ = brace_block(body, m.end())
        entries = split_top(blk)
        # Which h_ columns the expected values line up with.
        am = re.search(r"actual\[\{[^}]*\}\]\s*=\s*(\{[^;]*\}|h_\w+\[i\]);", body)
        if am:
            targets = re.findall(r"(h_\w+)\[i\]", am.group(1))
        else:
            targets = re.findall(r"EXPECT_NEAR\((h_\w+)\[i\],\s*\(?expected", body)
        tol = 0.0
        tm = re.search(r"EXPECT_NEAR\([^;]*,\s*([0-9.eE-]+)f?\)", body)
        if tm:
            tol = float(tm.group(1))
        for e in entries:
            kv = split_top(strip_braces(e))
            key = [num(x) for x in split_top(strip_braces(kv[0]))]
            vv = kv[1]
            values = [num(x) for x in split_top(strip_braces(vv))] if vv.strip().startswith("{") else [num(vv)]
            for tname, v in zip(targets, values):
                expects.append({"key": key, "column": hcol[tname], "value": v, "tol": tol})
    # Form 2: per-key if / else blocks inside the check loop.
    for im in re.finditer(r"if \(((?:h_key\d\[i\] == -?\d+(?:\s*&&\s*)?)+)\)\s*\{", body):
        conds = re.findall(r"h_key(\d)\[i\] == (-?\d+)", im.group(1))
        key = [int(v) for _, v in sorted(conds)]
        blk, end = brace_block(body, im.end() - 1)
        branches = [(key, blk)]
        em = re.match(r"\s*else\s*\{", body[end:])
        if em:
            eblk, _ = brace_block(body, end + em.end() - 1)
            tuples = sorted(set(zip(*[a["values"] for a in case["keys"]])))
            others = [list(t) for t in tuples if list(t) != key]
            if len(others) == 1:
                branches.append((others[0], eblk))
        for k, b in branches:
            for x in re.finditer(r"EXPECT_(EQ|NEAR)\((h_\w+)\[i\],\s*([-0-9.eE]+)f?(?:,\s*([0-9.eE-]+)f?)?\)", b):
                expects.append({"key": k, "column": hcol[x.group(2)], "value": num(x.group(3)),
                                "tol": float(x.group(4)) if x.group(4) else 0.0})
    # Form 3: single-row EXPECTs on index 0.
    for x in re.finditer(r"EXPECT_(EQ|NEAR)\((h_\w+)\[0\],\s*([-0-9.eE]+)f?(?:,\s*([0-9.eE-]+)f?)?\)", body):
        expects.append({"row": 0, "column": hcol[x.group(2)], "value": num(x.group(3)),
                        "tol": float(x.group(4)) if x.group(4) else 0.0})
    case["expects"] = expects
    if not expects:
        case["notes"].append("no literal expectations found")
    return case


def main() -> None:
    text = SRC.read_text()
    cases = []
    starts = [m for m in re.finditer(r"TEST_P\(GroupbyMultiKeysTest,\s*(\w+)\)\s*\{", text)]
    for m in starts:
        body, _ = brace_block(text, m.end() - 1)
        cases.append(parse_case(m.group(1), body))
    doc = {
        "source": "src/cuda/tests/groupby/groupby_multikeys_test.cu",
        "generator": "tests/golden/make_golden.py",
        "cases": cases,
    }
    OUT.write_text(json.dumps(doc, indent=1))
    ok = sum(1 for c in cases if c["ok"] and c.get("expects"))
    print(f"{len(cases)} cases, {ok} with inputs and expectations -> {OUT}")


if __name__ == "__main__":
    main()
