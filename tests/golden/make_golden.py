"""Write kat_layout_n8.json: the known-answer cases of the reference's N = 8
layout tests (crates/pir/src/base_pir.rs:1281-1411,
test_set_transformed_entries_full_group, _full_g_subgroup and
_small_subgroup), read from the reference's source text.

Each case is one database of a single non-zero entry (1 or X at entry
`index`) and the rows the reference expects `set_transformed_entries` to
store, as coefficients in {0, 1, -1} before the factor 1 / `factor` mod t and
the transform that assert_correctly_preprocessed applies (base_pir.rs:1292-1304).

Run with DNSPIR_REFERENCE naming a checkout of the reference (the directory
holding crates/pir); the JSON is committed and the tests read only the JSON:

    DNSPIR_REFERENCE=<path to the reference checkout> python tests/golden/make_golden.py
"""
import json
import os
import re

REF = os.environ.get("DNSPIR_REFERENCE")
SRC = os.path.join(REF or "", "crates", "pir", "src", "base_pir.rs")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "kat_layout_n8.json")
TESTS = ("test_set_transformed_entries_full_group", "test_set_transformed_entries_full_g_subgroup",
         "test_set_transformed_entries_small_subgroup")
VALUE = {"zero": 0, "one": 1, "neg_one": -1}
CASE = re.compile(r"set_transformed_entries\(\(0\.\.(\d+)\)\.map\(\|i\| if i == (\d+) \{ R\.(one|canonical_gen)\(\) \} "
                  r"else \{ R\.zero\(\) \}\)\);(.*?)assert_correctly_preprocessed\(&\[(.*?)\], &db\);", re.S)


def parse_rows(text):
    rows = [[VALUE[v] for v in re.findall(r"Zt\.(zero|one|neg_one)\(\)", r)] for r in re.findall(r"\[([^\[\]]*)\]", text)]
    rep = re.search(r"\]\s*;\s*(\d+)\s*$", text.strip())
    if rep:  # [row; k]
        assert len(rows) == 1
        rows = rows * int(rep.group(1))
    return rows


def main():
    if not REF:
        raise SystemExit("set DNSPIR_REFERENCE to the reference checkout (the directory holding crates/pir)")
    src = open(SRC).read()
    out = {"source": "crates/pir/src/base_pir.rs:1281-1411", "t": 1025, "tests": {}}
    for name in TESTS:
        i = src.index("fn " + name + "(")
        body = src[i:src.index("\n}\n", i)]
        factor = int(re.search(r"int_hom\(\)\.map\((\d+)\)", body).group(1))
        sub = re.search(r"IndexGroup::subgroup_of_size\(N, (\d+)\)", body)
        order = int(sub.group(1)) if sub else 8  # IndexGroup::full_group(N), N = 8
        cases = []
        for m in CASE.finditer(body):
            count, index, poly, _, rows = m.groups()
            cases.append({"count": int(count), "index": int(index), "entry": "1" if poly == "one" else "X",
                          "rows": parse_rows("[" + rows + "]" if ";" not in rows else rows)})
        assert len(cases) == 3, name
        out["tests"][name] = {"log2n": 3, "order": order, "factor": factor, "cases": cases}
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print("wrote", OUT)


if __name__ == "__main__":
    main()
