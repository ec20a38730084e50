"""The 6502opt command line against the reference CLI's behaviour
(cmd/6502opt/main.go): verify-jsonl (:386-463), the WriteJSON array of
`enumerate --output` (pkg/result/output.go:21-35), `target
--max-candidate` (:130) and the resume watermark of `enumerate
--checkpoint`.  GPU tests run the built CLI on the device; the others need
no GPU."""
import io
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG_DIR
from m6502 import _lib
from m6502 import inst as I
from m6502.result import jsonl_line, make_rule, write_json

CLI = os.path.join(PKG_DIR, "bin", "6502opt")


@pytest.fixture(scope="module")
def cli():
    if not os.path.exists(CLI):
        subprocess.run(["make", "-s", "-C", PKG_DIR, "cli"], check=True)
    return CLI


def run(cli, *args, **kw):
    return subprocess.run([cli, *args], capture_output=True, text=True, timeout=kw.pop("timeout", 900), **kw)


# Go's json.Encoder with SetIndent("", "  ") on []JSONRule, written out by
# hand: dead_flags is omitted when empty (omitempty), a trailing newline ends
# the document.
GO_LAYOUT = """[
  {
    "source": [
      "ROL A",
      "AND #$FE"
    ],
    "replacement": [
      "ASL A"
    ],
    "bytes_saved": 2,
    "cycles_saved": 2
  },
  {
    "source": [
      "CMP #$10",
      "LDA #$00"
    ],
    "replacement": [
      "LDA #$00"
    ],
    "bytes_saved": 2,
    "cycles_saved": 2,
    "dead_flags": "C,Z,N"
  }
]
"""


def test_write_json_layout():
    rules = [make_rule(I.parse_assembly("ROL A : AND #$FE"), I.parse_assembly("ASL A")),
             make_rule(I.parse_assembly("CMP #$10 : LDA #$00"), I.parse_assembly("LDA #$00"), dead_flags=0x83)]
    buf = io.StringIO()
    write_json(buf, rules)
    assert buf.getvalue() == GO_LAYOUT
    empty = io.StringIO()
    write_json(empty, [])
    assert empty.getvalue() == "[]\n"


def test_target_max_candidate_above_two_is_an_error(cli):
    r = run(cli, "target", "TXA : TAX", "--max-candidate", "3")
    assert r.returncode == 1
    assert "length 1..2" in r.stderr


def test_search_mirror_refuses_long_candidates():
    from m6502.search import Config, Run, SearchSingle
    with pytest.raises(ValueError):
        SearchSingle(I.parse_assembly("TXA : TAX"), 3)
    with pytest.raises(ValueError):
        Run(Config(MaxTargetLen=4))


@pytest.mark.gpu
def test_target_command(cli):
    r = run(cli, "target", "TXA : TAX")
    assert r.returncode == 0, r.stderr
    assert "Replacement: TXA (-1 bytes, -2 cycles)" in r.stdout
    r = run(cli, "target", "CMP #$10 : LDA #$00", "--dead-flags", "all")
    assert r.returncode == 0, r.stderr
    assert "Replacement: LDA #$00" in r.stdout


@pytest.mark.gpu
def test_search_mirror_length2_candidates(engine):
    """SearchSingle with MaxCandLen 2 finds a length-2 rewrite where no
    length-1 candidate exists, as the Go worker's candLen loop does
    (pkg/search/worker.go:122-176); with MaxCandLen 1 it finds none."""
    from m6502.search import SearchSingle
    import oracle
    targets = oracle.draw_targets(1, 3, 64)
    want, _ = oracle.search_go(targets, dead=0, max_cand_len=2)
    two = [(t, c) for t, c, _ in want if len(c) == 2]
    assert two, "the seeded draw holds a target whose best rewrite has two instructions"
    ti, c = two[0]
    t = [int(x) for x in targets[ti]]
    r2 = SearchSingle(t, 2, engine=engine)
    assert r2 is not None and r2.Replacement == list(c)
    assert SearchSingle(t, 1, engine=engine) is None


@pytest.mark.gpu
def test_enumerate_output_is_write_json(cli, engine, tmp_path):
    """`enumerate --output` (Go semantics) writes the same document as the
    Python WriteJSON mirror does for the engine's rules, byte for byte."""
    out = tmp_path / "rules.json"
    r = run(cli, "enumerate", "--max-target", "2", "--first-op-start", "0", "--first-op-end", "40",
            "--output", str(out))
    assert r.returncode == 0, r.stderr
    text = out.read_text()
    rules, _ = engine.enumerate(2, semantics=_lib.SEM_GO, sweep=_lib.SWEEP_REFERENCE, first=0, last=40)
    tab = I.insn_table(_lib.SEM_CUDA)
    mine = []
    for row in sorted(rules, key=lambda x: (int(x["target"]), int(x["cand_len"]), tuple(x["cand"]))):
        tid = int(row["target"])
        t = [int(tab[tid // 2863]), int(tab[tid % 2863])]
        mine.append(make_rule(t, [int(x) for x in row["cand"][:row["cand_len"]]], _lib.SEM_GO,
                              int(row["dead_flags"])))
    mine.sort(key=lambda x: (-x.BytesSaved, -x.CyclesSaved))   # a stable sort, as Table.Rules
    buf = io.StringIO()
    write_json(buf, mine)
    assert len(json.loads(text)) == len(rules) > 0
    assert text == buf.getvalue()


@pytest.fixture(scope="module")
def full_jsonl(cli, tmp_path_factory):
    """The JSONL of a full length-2 enumeration (CUDA semantics, reduced
    sweep: the reference pipeline's 1,078,897 rules)."""
    path = tmp_path_factory.mktemp("jsonl") / "len2.jsonl"
    with open(path, "w") as f:
        r = subprocess.run([cli, "enumerate", "--jsonl", "--max-target", "2", "--sweep", "reference"],
                           stdout=f, stderr=subprocess.PIPE, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    return path


@pytest.mark.gpu
def test_verify_jsonl_accepts_a_full_enumeration(cli, full_jsonl):
    with open(full_jsonl) as f:
        n = sum(1 for _ in f)
    assert n == 1_078_897
    r = run(cli, "verify-jsonl", str(full_jsonl), "--sweep", "reference")
    assert r.returncode == 0, r.stderr[-2000:]
    assert f"Verification complete: {n} total, {n} passed, 0 failed, 0 skipped" in r.stdout


@pytest.mark.gpu
def test_verify_jsonl_rejects_a_corrupted_rule(cli, full_jsonl, tmp_path):
    """One rule's replacement is swapped for a non-equivalent instruction and
    one line is not JSON: the command prints FAIL for the first, skips the
    second and exits non-zero."""
    bad = tmp_path / "bad.jsonl"
    with open(full_jsonl) as f, open(bad, "w") as g:
        for i, line in enumerate(f):
            if i >= 20000:
                break
            if i == 1234:
                d = json.loads(line)
                d["replacement_asm"] = "INX" if d["replacement_asm"] != "INX" else "INY"
                line = json.dumps(d) + "\n"
            if i == 1235:
                line = "{not json\n"
            g.write(line)
    r = run(cli, "verify-jsonl", str(bad), "--sweep", "reference")
    assert r.returncode != 0
    assert "[1235] FAIL:" in r.stdout
    assert "19998 passed, 1 failed, 1 skipped" in r.stdout


@pytest.mark.gpu
def test_verify_jsonl_reports_undecided(cli, tmp_path):
    """A rule whose full sweep exceeds the engine's per-cone cap is reported
    UNDECIDED, not FAIL, and the command exits non-zero.  Here the final A
    depends on A, X, Y, M, S0 and carry (a cone of 2^41 states under the full
    sweep, above the 2^34 cap); the replacement appends a NOP, so no sampled
    state differs."""
    src = "ADC M : STA M : TXA : ADC M : STA M : TYA : ADC M : STA M : PLA : ADC M"
    f = tmp_path / "u.jsonl"
    f.write_text(json.dumps({"source_asm": src, "replacement_asm": src + " : NOP"}) + "\n")
    r = run(cli, "verify-jsonl", str(f), "--sweep", "full")
    assert r.returncode != 0
    assert "[1] UNDECIDED:" in r.stdout
    assert "0 passed, 0 failed, 0 skipped, 1 undecided" in r.stdout


@pytest.mark.gpu
def test_enumerate_checkpoint_resume(cli, engine, tmp_path):
    """--checkpoint: a run resumed from a watermark emits exactly the rules of
    the first-ops not yet done, and leaves the watermark past the end."""
    ck = tmp_path / "ck"
    ck.write_text("2 100\n")
    r = run(cli, "enumerate", "--jsonl", "--max-target", "2", "--first-op-start", "0", "--first-op-end", "230",
            "--sweep", "reference", "--checkpoint", str(ck))
    assert r.returncode == 0, r.stderr
    assert "resuming at target length 2, first-op 100" in r.stderr
    got = sorted(json.dumps(json.loads(x), sort_keys=True) for x in r.stdout.splitlines() if x.startswith("{"))
    rules, _ = engine.enumerate(2, semantics=_lib.SEM_CUDA, sweep=_lib.SWEEP_REFERENCE, first=100, last=230)
    tab = I.insn_table(_lib.SEM_CUDA)
    want = []
    for row in rules:
        tid = int(row["target"])
        want.append(json.dumps(json.loads(jsonl_line([int(tab[tid // 2863]), int(tab[tid % 2863])], row, 0)),
                               sort_keys=True))
    assert got == sorted(want) and len(got) > 0
    assert ck.read_text().split() == ["3", "0"]
    r = run(cli, "enumerate", "--jsonl", "--max-target", "2", "--first-op-start", "0", "--first-op-end", "230",
            "--sweep", "reference", "--checkpoint", str(ck))
    assert r.returncode == 0 and not any(x.startswith("{") for x in r.stdout.splitlines())
