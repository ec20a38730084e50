"""`6502opt export -f go` (cmd/6502opt/main.go:147-194): a rules JSON file in
WriteJSON's layout becomes Go peephole code in WriteGoCode's layout
(pkg/result/output.go:47-75).  As in the reference, the dead_flags of the
JSON are not carried into the code, and rules that do not parse are skipped
with a message on stderr."""
import json
import os
import subprocess

import pytest

from conftest import PKG_DIR

CLI = os.path.join(PKG_DIR, "bin", "6502opt")


@pytest.fixture(scope="module")
def cli():
    if not os.path.exists(CLI):
        subprocess.run(["make", "-s", "-C", PKG_DIR, "cli"], check=True)
    return CLI


def expected_go(rules):
    q = lambda s: '"' + s.replace("\\", "\\\\").replace('"', '\\"') + '"'  # noqa: E731
    out = ["package peephole\n\n// Generated by 6502opt. DO NOT EDIT.\n\n",
           "type PeepholeRule struct {\n\tSource      []string\n\tReplacement []string\n",
           "\tBytesSaved  int\n\tCyclesSaved int\n\tDeadFlags   string\n}\n\n", "var Rules = []PeepholeRule{\n"]
    for r in rules:
        out.append(f"\t// {' : '.join(r['source'])} -> {' : '.join(r['replacement'])} "
                   f"(-{r['bytes_saved']} bytes, -{r['cycles_saved']} cycles)\n")
        out.append("\t{Source: []string{" + ", ".join(q(x) for x in r["source"]) + "}, Replacement: []string{"
                   + ", ".join(q(x) for x in r["replacement"]) + "}, "
                   f"BytesSaved: {r['bytes_saved']}, CyclesSaved: {r['cycles_saved']}}},\n")
    out.append("}\n")
    return "".join(out)


def test_export_go(cli, tmp_path):
    rules = [
        {"source": ["TXA", "TAX"], "replacement": ["TXA"], "bytes_saved": 1, "cycles_saved": 2},
        {"source": ["ROL A", "AND #$FE"], "replacement": ["ASL A"], "bytes_saved": 2, "cycles_saved": 2},
        {"source": ["CMP #$00", "CLC"], "replacement": ["CLC"], "bytes_saved": 2, "cycles_saved": 2,
         "dead_flags": "Z,N"},
        {"source": ["BOGUS"], "replacement": ["NOP"], "bytes_saved": 1, "cycles_saved": 0},
    ]
    f = tmp_path / "rules.json"
    f.write_text(json.dumps(rules, indent=2))
    run = subprocess.run([cli, "export", "-f", "go", str(f)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stderr
    assert run.stdout == expected_go(rules[:3])
    assert "skipping rule (bad source)" in run.stderr


def test_export_rejects_unknown_format(cli, tmp_path):
    f = tmp_path / "rules.json"
    f.write_text("[]")
    run = subprocess.run([cli, "export", "-f", "c", str(f)], capture_output=True, text=True, timeout=60)
    assert run.returncode != 0 and "unknown format" in run.stderr
