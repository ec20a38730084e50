"""Rules and their output formats (mirror of pkg/result and the CUDA JSONL).

* ``write_json`` -- the Go CLI's pretty JSON array (pkg/result/output.go:12-35),
  rules sorted by bytes saved then cycles saved (table.go:37-50).
* ``jsonl_line`` -- one line of the CUDA pipeline's JSONL
  (cuda/6502_search_v2.cu:912-930), read back by ``verify-jsonl``.
"""
import ctypes
import json
from dataclasses import dataclass, field
from typing import List

import numpy as np

from . import _lib
from .inst import Disassemble, SeqByteSize, SeqCycles


@dataclass
class Rule:
    Source: List[int]
    Replacement: List[int]
    BytesSaved: int
    CyclesSaved: int
    DeadFlags: int = 0
    extra: dict = field(default_factory=dict)


def DeadFlagDesc(mask):
    """pkg/result/output.go:77-101."""
    if mask == 0:
        return ""
    if mask == 0xFF:
        return "all"
    names = [(0x01, "C"), (0x02, "Z"), (0x04, "I"), (0x08, "D"), (0x40, "V"), (0x80, "N")]
    return ",".join(n for b, n in names if mask & b)


def make_rule(source, replacement, semantics=_lib.SEM_GO, dead_flags=0):
    return Rule(list(source), list(replacement),
                SeqByteSize(source, semantics) - SeqByteSize(replacement, semantics),
                SeqCycles(source) - SeqCycles(replacement), dead_flags)


def sort_rules(rules):
    """Table.Rules order: bytes saved desc, then cycles saved desc."""
    return sorted(rules, key=lambda r: (-r.BytesSaved, -r.CyclesSaved))


def write_json(fp, rules):
    out = []
    for r in rules:
        d = {"source": [Disassemble(i) for i in r.Source],
             "replacement": [Disassemble(i) for i in r.Replacement],
             "bytes_saved": r.BytesSaved, "cycles_saved": r.CyclesSaved}
        desc = DeadFlagDesc(r.DeadFlags)
        if desc:
            d["dead_flags"] = desc
        out.append(d)
    fp.write(json.dumps(out, indent=2) + "\n")


def jsonl_line(target, rule_row, run_dead_flags=0):
    """Formats one device rule (RULE_DTYPE row) against its target sequence."""
    t = _lib.u16(target)
    r = _lib.Rule()
    r.target = int(rule_row["target"])
    r.cand_len = int(rule_row["cand_len"])
    r.dead_flags = int(rule_row["dead_flags"])
    for i in range(3):
        r.cand[i] = int(rule_row["cand"][i])
    buf = ctypes.create_string_buffer(512)
    n = _lib.lib().m6502_format_jsonl(_lib.ptr(t, ctypes.c_uint16), len(t), ctypes.byref(r),
                                      run_dead_flags, buf, 512)
    if n < 0:
        raise ValueError("bad rule")
    return buf.value.decode()


def rule_pairs(rules, targets):
    """Set of (target tuple, replacement tuple, dead_flags) for set-equality tests."""
    targets = np.asarray(targets)
    out = set()
    for r in rules:
        t = tuple(int(x) for x in targets[int(r["target"])])
        c = tuple(int(x) for x in r["cand"][:int(r["cand_len"])])
        out.add((t, c, int(r["dead_flags"])))
    return out
