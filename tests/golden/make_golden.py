"""Regenerate the golden fixtures of tests/golden/ from the reference tree.

Run with the root of a reference checkout as the one required argument:

    python tests/golden/make_golden.py REFERENCE_ROOT

Fixtures written (small, committed):
  routing.json — the routing workload's input rows (examples/workloads/routing/
                 links.tsv) and the three lines its CI test pins
                 (crates/strata-cli/tests/workloads.rs:26-32).
  tc_example.json — examples/edges.tsv rows (the tc_tsv.strata input).
  aml.json     — the AML workload's four TSV inputs (examples/workloads/aml/)
                 and the four lines its CI test pins
                 (crates/strata-cli/tests/workloads.rs:17-23).
The tests never read the reference tree; they read these files.
"""
import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def tsv_rows(p: Path):
    rows = []
    for line in p.read_text().splitlines():
        line = line.rstrip("\r")
        if line:
            rows.append(line.split("\t"))
    return rows


def main(ref: Path) -> None:
    links = tsv_rows(ref / "examples/workloads/routing/links.tsv")
    pinned = []
    src = (ref / "crates/strata-cli/tests/workloads.rs").read_text()
    for line in src.splitlines():
        line = line.strip()
        if line.startswith('"route('):
            pinned.append(line.strip('",'))
    (HERE / "routing.json").write_text(json.dumps({
        "source": "examples/workloads/routing/links.tsv; pinned lines from "
                  "crates/strata-cli/tests/workloads.rs:26-32",
        "rows": links,
        "queries": [["n0_0", "n7_7"], ["n0_0", "n4_4"], ["n7_7", "n0_0"]],
        "pinned": pinned,
    }, indent=0))
    edges = tsv_rows(ref / "examples/edges.tsv")
    (HERE / "tc_example.json").write_text(json.dumps({
        "source": "examples/edges.tsv (input of examples/tc_tsv.strata)",
        "rows": edges,
    }, indent=0))
    aml = ref / "examples/workloads/aml"
    src_lines = (ref / "crates/strata-cli/tests/workloads.rs").read_text().splitlines()
    start = next(i for i, l in enumerate(src_lines) if l.strip() == '"aml",')
    aml_pinned = []
    for line in src_lines[start + 1:]:
        t = line.strip()
        if t.startswith("),"):
            break
        if t.startswith('"') and "::" in t:
            aml_pinned.append(json.loads(t.rstrip(",").replace("\\u{2202}", "\u2202").replace("\\u{2192}", "\u2192")))
    (HERE / "aml.json").write_text(json.dumps({
        "source": "examples/workloads/aml/{companies,ownership,sanctions,flags}.tsv; pinned lines from "
                  "crates/strata-cli/tests/workloads.rs:17-23",
        "entity": tsv_rows(aml / "companies.tsv"),
        "owns": tsv_rows(aml / "ownership.tsv"),
        "sanctioned": tsv_rows(aml / "sanctions.tsv"),
        "flag": tsv_rows(aml / "flags.tsv"),
        "queries": [["investigate", "g0_hold"], ["cleared", "indie0"], ["cleared", "indie7"]],
        "pinned": aml_pinned,
    }, indent=0, ensure_ascii=False))
    print(f"routing: {len(links)} rows, pinned {pinned}; tc_example: {len(edges)} rows; aml pinned {aml_pinned}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py REFERENCE_ROOT")
    main(Path(sys.argv[1]))
