"""Regenerate tests/golden/golden.json from the reference's test data.

Run once where a checkout of the reference module exists, passing its path
with --ref (required).  The output is committed, so the tests never read the reference.

What it records:
  * the four byte-exact golden blocks of testdata/*.bin together with the
    inputs and flags the reference packs them from
    (format_conformance_test.go:695-754);
  * the reference's fuzz corpus inputs for corrupt-block APIs
    (testdata/fuzz/*), parsed from the Go fuzz v1 text format;
  * the known answers printed by the reference's Example functions
    (example_test.go), written out as (inputs, flags, expected) records.
"""
import argparse
import ast
import json
import os


def golden_inputs():
    # format_conformance_test.go:695-725
    bw8 = [128 + i for i in range(128)]
    bw0 = [0] * 128
    delta = [i * 100 for i in range(128)]
    exc = list(range(128))
    for p in (5, 15, 25, 35, 45, 55, 65, 75, 85, 95):
        exc[p] = 0x10000000 + p
    return [
        ("plain_128_bw8", "plain_128_bw8.bin", bw8, 0),
        ("plain_128_bw0", "plain_128_bw0.bin", bw0, 0),
        ("delta_128", "delta_128.bin", delta, 1),
        ("exceptions_128", "exceptions_128.bin", exc, 0),
    ]


def parse_go_fuzz(path):
    """Go fuzz corpus v1: one header line, then one Go literal per line."""
    with open(path, "r", encoding="latin-1") as f:
        lines = f.read().splitlines()
    assert lines[0] == "go test fuzz v1", path
    vals = []
    for ln in lines[1:]:
        ln = ln.strip()
        if ln.startswith("[]byte(") and ln.endswith(")"):
            lit = ln[len("[]byte("):-1]
            vals.append(list(ast.literal_eval("b" + lit)))
        else:
            vals.append(ln)
    return vals


def examples():
    # example_test.go known answers (Output: blocks)
    out = []
    out.append({"name": "ExamplePackUint32", "kind": "pack32_len", "flag": 0,
                "values": [10, 20, 30, 40, 50], "want": 18})
    vals = [100000 + i * 4 for i in range(128)]
    out.append({"name": "ExamplePackUint32_delta/plain", "kind": "pack32_len", "flag": 0,
                "values": vals, "want": 200})
    out.append({"name": "ExamplePackUint32_delta/delta", "kind": "pack32_len", "flag": 1,
                "values": vals, "want": 136})
    vals = [4_000_000 + i % 16 for i in range(128)]
    vals[10] = 4_500_000
    vals[90] = 4_600_000
    for flag, want in ((0, 81), (2, 388), (4, 328), (6, 388)):
        out.append({"name": "ExamplePackUint32_flags/%d" % flag, "kind": "pack32_len",
                    "flag": flag, "values": vals, "want": want})
    out.append({"name": "ExamplePackUint32_append", "kind": "append32_lens", "flag": 16,
                "blocks": [[1, 2, 3, 4], [100, 200, 300, 400]], "want": [15, 17]})
    out.append({"name": "ExamplePackUint32_noInPlace", "kind": "append32_total", "flag": 16,
                "blocks": [[500 + i * 3 for i in range(128)]] * 3, "want": 588})
    out.append({"name": "ExampleBlockLength_skipBlocks", "kind": "skip_blocks", "flag": 16,
                "blocks": [[1, 2, 3], [100, 200, 300]], "want": 13})
    out.append({"name": "ExampleHeader", "kind": "header32", "flag": 1 | 4,
                "values": [i * 10 for i in range(128)],
                "want": {"count": 128, "bit_width": 8, "exc_count": 0, "delta": True, "for": False}})
    out.append({"name": "ExamplePackUint64", "kind": "pack64_len", "flag": 0,
                "values": [1_000_000_000_000, 1_000_000_000_001, 1_000_000_000_002], "want": 19})
    out.append({"name": "ExampleNewUint32_delta", "kind": "pack32_len", "flag": 1,
                "values": [1000 + i * 4 for i in range(128)], "want": 170})
    out.append({"name": "ExampleMaxBlockLength32", "kind": "max32",
                "want": {"0": 1018, "4": 520, "6": 516, "2": 1014}})
    out.append({"name": "ExampleMaxBlockLength64", "kind": "max64",
                "want": {"0": 2038, "4": 1042}})
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="checkout of the reference module (its testdata/ is read)")
    ap.add_argument("--out", default=os.path.join(os.path.dirname(__file__), "golden.json"))
    a = ap.parse_args()
    td = os.path.join(a.ref, "testdata")
    blocks = []
    for name, fn, values, flag in golden_inputs():
        with open(os.path.join(td, fn), "rb") as f:
            data = f.read()
        blocks.append({"name": name, "file": "testdata/" + fn, "flag": flag,
                       "values": values, "packed_hex": data.hex()})
    fuzz = []
    fdir = os.path.join(td, "fuzz")
    for sub in sorted(os.listdir(fdir)):
        for fn in sorted(os.listdir(os.path.join(fdir, sub))):
            fuzz.append({"target": sub, "file": fn,
                         "args": parse_go_fuzz(os.path.join(fdir, sub, fn))})
    doc = {"source": "Akron/utlpfor testdata + example_test.go",
           "golden_blocks": blocks, "fuzz_corpus": fuzz, "examples": examples()}
    with open(a.out, "w") as f:
        json.dump(doc, f, separators=(",", ":"))
        f.write("\n")
    print("wrote", a.out)


if __name__ == "__main__":
    main()
