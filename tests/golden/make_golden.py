"""Generates the golden fixtures of tests/golden from the reference's own
host code (oracle/_ref/libref6502.so, built by `make -C oracle ref` from the
reference sources).  Run from the repository root:

    python tests/golden/make_golden.py

Fixtures written (all small):
  exec_vectors.npz     2,863 instructions x 6 seeded random states: inputs and
                       outputs of h_exec_instruction (cuda/6502_common.h:237-314)
  prune.json           population count and SHA-256 of should_prune over all
                       8,196,769 length-2 sequences in CUDA order
                       (cuda/6502_search_v2.cu:600-622)
  config1.json         the 256 seeded length-2 targets (seed 0) and the rule
                       sets + stage counts of the reference pipeline
                       (cuda/6502_search_v2.cu:848-977) for dead-flags 0x00 and
                       0x01, and for 0xC3 / 0xFF on the first 64 targets that
                       have at most 12 MidCheck survivors (bounds the CPU time)
  pairs.json           (target, candidate, mask) pairs with the reference's
                       QC / MidCheck / ExhaustiveCheck verdicts
"""
import hashlib
import json
import os
import sys
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def ref_exec(state, insn):
    s = oracle.State(*state)
    oracle.ref().ref_exec(oracle.ctypes.byref(s), insn & 0xFF, insn >> 8)
    return s.tuple()


def seq_ptr(seq):
    a = np.ascontiguousarray(np.asarray(seq, dtype=np.uint16))
    return a, a.ctypes.data_as(oracle.ctypes.POINTER(oracle.ctypes.c_uint16)), len(a)


def ref_fp(seq):
    a, p, n = seq_ptr(seq)
    out = (oracle.ctypes.c_uint8 * 64)()
    oracle.ref().ref_fingerprint(p, n, out)
    return bytes(out)


def ref_qc(t, c, dead):
    a, b = ref_fp(t), ref_fp(c)
    for i in range(64):
        m = (~dead & 0xFF) if i % 8 == 3 else 0xFF
        if (a[i] ^ b[i]) & m:
            return False
    return True


def ref_mid(t, c, dead):
    ta, tp, tn = seq_ptr(t)
    ca, cp, cn = seq_ptr(c)
    return bool(oracle.ref().ref_midcheck(tp, tn, cp, cn, dead))


def ref_exh(t, c, dead):
    ta, tp, tn = seq_ptr(t)
    ca, cp, cn = seq_ptr(c)
    return bool(oracle.ref().ref_exhaustive(tp, tn, cp, cn, dead))


def main():
    assert oracle.ref_available(), "build the reference host code first: make -C oracle ref"
    tab = oracle.insn_table(oracle.SEM_CUDA)
    rng = np.random.default_rng(6502)

    # 1. executor
    t0 = time.time()
    states = rng.integers(0, 256, size=(len(tab), 6, 8), dtype=np.uint8)
    outs = np.zeros_like(states)
    for i, insn in enumerate(tab):
        for j in range(states.shape[1]):
            outs[i, j] = ref_exec(tuple(int(x) for x in states[i, j]), int(insn))
    np.savez_compressed(os.path.join(OUT, "exec_vectors.npz"), insns=tab, inputs=states, outputs=outs)
    print(f"exec_vectors: {time.time() - t0:.1f}s")

    # 2. pruner over all length-2 sequences
    t0 = time.time()
    bits = np.zeros(len(tab) * len(tab), dtype=np.uint8)
    seq = (oracle.ctypes.c_uint16 * 2)()
    R = oracle.ref()
    k = 0
    for a in tab:
        seq[0] = int(a)
        for b in tab:
            seq[1] = int(b)
            bits[k] = R.ref_should_prune(seq, 2)
            k += 1
    packed = np.packbits(bits)
    prune = {"pruned": int(bits.sum()), "kept": int(len(bits) - bits.sum()),
             "sha256_packbits": hashlib.sha256(packed.tobytes()).hexdigest()}
    json.dump(prune, open(os.path.join(OUT, "prune.json"), "w"), indent=1)
    print(f"prune: {prune} {time.time() - t0:.1f}s")

    # 3. config 1
    t0 = time.time()
    targets = oracle.draw_targets(0, 2, 256)
    cfg1 = {"seed": 0, "targets": targets.tolist(), "runs": {}}
    for dead in (0x00, 0x01, 0xC3, 0xFF):
        sel = np.arange(len(targets))
        if dead in (0xC3, 0xFF):
            # The reference's CPU sweep is slow for relaxed masks: keep the
            # first 64 targets with at most 12 MidCheck survivors each.
            keep = []
            for i in range(len(targets)):
                _, c = oracle.ref_search(targets[i:i + 1], dead=dead, stages=3, nthreads=1)
                if c["mid_hits"] <= 12:
                    keep.append(i)
                if len(keep) == 64:
                    break
            sel = np.array(keep)
        sub = targets[sel]
        rules, counts = oracle.ref_search(sub, dead=dead)
        cfg1["runs"][f"0x{dead:02X}"] = {
            "target_index": sel.tolist(), "counts": counts,
            "rules": sorted([[r[0], list(r[1])] for r in rules]),
            "jsonl": sorted(oracle.format_jsonl(sub[r[0]], r, dead) for r in rules)}
        print(f"config1 mask 0x{dead:02X}: {len(sub)} targets {len(rules)} rules {counts} {time.time() - t0:.1f}s")
    json.dump(cfg1, open(os.path.join(OUT, "config1.json"), "w"))

    # 4. pair verdicts: QC-passing candidates of seeded targets of length 1..3
    t0 = time.time()
    cands = [[int(c)] for c in tab]
    pool = []
    for tlen, seed, n in ((1, 11, 40), (2, 12, 40), (3, 13, 30)):
        for t in oracle.draw_targets(seed, tlen, n):
            pool.append([int(x) for x in t])
    examples = [("ROL A : AND #$FE", "ASL A"), ("ROR A : AND #$7F", "LSR A"),
                ("LDA M : EOR M", "LDA #$00"), ("BIT M : ADC #$00", "ADC #$00"), ("TXA : TAX", "TXA"),
                ("CLC : CLC", "CLC"), ("LDA #$00", "AND #$00"), ("LDA #$00", "EOR #$00"),
                ("PHA : PLA", "CMP #$00"), ("PHP : PLP", "CLV"), ("TXA : INX", "TXA : INX"),
                ("STX M : LDA M", "TXA : STX M"), ("PHA : TXA : PLA", "LDA M"),
                ("SEC : SBC #$01", "CLC : ADC #$FF"), ("PHA : PHA : PLA", "PHA : TAY")]
    pairs = []
    for dead in (0x00, 0x01, 0xC3, 0xFF):
        picked = []
        for t in pool:
            hits = [c for c in cands if ref_qc(t, c, dead) and sweep_states(t, c) <= (1 << 17)]
            rng.shuffle(hits)
            picked += [(t, c) for c in hits[:3]]
            nz = [c for c in cands if not ref_qc(t, c, dead)]
            picked.append((t, nz[int(rng.integers(len(nz)))]))
        for a, b in examples:
            picked.append((list(oracle_parse(a)), list(oracle_parse(b))))

        def verdict(tc):
            t, c = tc
            return {"t": t, "c": c, "dead": dead, "qc": ref_qc(t, c, dead), "mid": ref_mid(t, c, dead),
                    "exh": ref_exh(t, c, dead)}

        with ThreadPoolExecutor(max_workers=os.cpu_count()) as ex:
            pairs += list(ex.map(verdict, picked))
        print(f"pairs mask 0x{dead:02X}: {len(picked)} {time.time() - t0:.1f}s")
    json.dump(pairs, open(os.path.join(OUT, "pairs.json"), "w"))
    print("done")


def sweep_states(t, c):
    """States of the reference sweep of a pair (bounds the fixture's CPU time)."""
    reads = 0
    for x in list(t) + list(c):
        reads |= int(oracle.lib().or_op_reads(x & 0xFF))
    k = bin(reads & 0xFC).count("1")
    return 512 * (32 ** k if k >= 3 else 256 ** k)


def oracle_parse(text):
    out = []
    for part in text.split(":"):
        v = oracle.ctypes.c_uint16()
        assert oracle.lib().or_parse_insn(part.strip().encode(), oracle.ctypes.byref(v)) == 0, part
        out.append(v.value)
    return out


if __name__ == "__main__":
    main()
