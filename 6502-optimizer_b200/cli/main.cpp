// 6502opt -- command-line driver over libm6502gpu.so, mirroring the
// reference CLI (cmd/6502opt/main.go) and the CUDA pipeline's flags
// (cuda/6502_search_v2.cu:768-789):
//
//   6502opt enumerate [--max-target N] [--output FILE] [--dead-flags M] [-v]
//                     [--jsonl] [--semantics go|cuda] [--sweep full|reference]
//                     [--first-op-start A] [--first-op-end B] [--no-exhaust]
//                     [--gpu-id N] [--checkpoint FILE] [--workers N]
//   6502opt target "LDA #$00 : TAX" [--max-candidate N<=2] [--dead-flags M] [-v]
//   6502opt verify-jsonl FILE [--dead-flags M] [-v] [--sweep full|reference]
//   6502opt stoke --target "PHA : TXA : PLA" [--chains N] [--iterations I] [--decay D]
//                 [--output FILE] [-v] [--dead-flags M] [--cost ref|hamming] [--seed S]
//
// All checking runs on the GPU through the C ABI; there is no CPU path.
#include <algorithm>
#include <cctype>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <iterator>
#include <map>
#include <string>
#include <vector>

#include "m6502.h"

namespace {

struct Args {
    std::vector<std::string> pos;
    std::map<std::string, std::string> kv;
    bool has(const std::string& k) const { return kv.count(k) != 0; }
    std::string get(const std::string& k, const std::string& d) const {
        auto it = kv.find(k);
        return it == kv.end() ? d : it->second;
    }
    long num(const std::string& k, long d) const { return has(k) ? std::strtol(kv.at(k).c_str(), nullptr, 0) : d; }
};

const char* kFlagsNoValue[] = {"-v", "--verbose", "--jsonl", "--no-exhaust", "--help", "-h"};

Args parse_args(int argc, char** argv, int start) {
    Args a;
    for (int i = start; i < argc; i++) {
        std::string s = argv[i];
        bool novalue = false;
        for (const char* f : kFlagsNoValue) novalue = novalue || s == f;
        if (novalue) { a.kv[s] = "1"; continue; }
        if (s.rfind("--", 0) == 0 || (s.size() == 2 && s[0] == '-')) {
            size_t eq = s.find('=');
            if (eq != std::string::npos) a.kv[s.substr(0, eq)] = s.substr(eq + 1);
            else if (i + 1 < argc) a.kv[s] = argv[++i];
            else a.kv[s] = "";
            continue;
        }
        a.pos.push_back(s);
    }
    return a;
}

// parseDeadFlags (cmd/6502opt/main.go:285-299): none, all, or hex.
bool parse_dead(const std::string& s0, uint8_t* out) {
    std::string s;
    for (char c : s0) s += (char)std::tolower((unsigned char)c);
    if (s == "none" || s.empty()) { *out = 0; return true; }
    if (s == "all") { *out = 0xFF; return true; }
    if (s.rfind("0x", 0) == 0) s = s.substr(2);
    char* end = nullptr;
    unsigned long v = std::strtoul(s.c_str(), &end, 16);
    if (s.empty() || *end || v > 0xFF) return false;
    *out = (uint8_t)v;
    return true;
}

// DeadFlagDesc (pkg/result/output.go:77-101).
std::string dead_desc(uint8_t m) {
    if (!m) return "";
    if (m == 0xFF) return "all";
    const std::pair<uint8_t, const char*> f[] = {{0x01, "C"}, {0x02, "Z"}, {0x04, "I"}, {0x08, "D"}, {0x40, "V"}, {0x80, "N"}};
    std::string s;
    for (auto& p : f)
        if (m & p.first) { if (!s.empty()) s += ","; s += p.second; }
    return s;
}

std::string disasm(uint16_t insn) {
    char b[32];
    m6502_disasm(insn, b, sizeof b);
    return b;
}

std::string disasm_seq(const uint16_t* s, int n) {
    std::string r;
    for (int i = 0; i < n; i++) { if (i) r += " : "; r += disasm(s[i]); }
    return r;
}

m6502_ctx* open_ctx(int device) {
    m6502_opts o{};
    o.device = device;
    m6502_ctx* ctx = nullptr;
    int rc = m6502_create(&ctx, &o);
    if (rc != M6502_OK) {
        std::fprintf(stderr, "error: cannot open GPU %d (code %d): the engine needs a CUDA device\n", device, rc);
        std::exit(2);
    }
    return ctx;
}

void die(m6502_ctx* ctx, int rc, const char* what) {
    std::fprintf(stderr, "error: %s failed (%d): %s\n", what, rc, ctx ? m6502_last_error(ctx) : "");
    std::exit(1);
}

struct OutRule {
    std::vector<uint16_t> src, rep;
    int bytes_saved, cycles_saved;
    uint8_t dead;
};

std::string json_str(const std::string& s) {
    std::string r = "\"";
    for (char c : s) {
        if (c == '"' || c == '\\') { r += '\\'; r += c; }
        else r += c;
    }
    return r + "\"";
}

// WriteJSON (pkg/result/output.go:21-35): pretty array, 2-space indent.
void write_json(std::ostream& os, const std::vector<OutRule>& rules) {
    if (rules.empty()) { os << "[]\n"; return; }
    os << "[\n";
    for (size_t i = 0; i < rules.size(); i++) {
        const OutRule& r = rules[i];
        os << "  {\n    \"source\": [\n";
        for (size_t k = 0; k < r.src.size(); k++)
            os << "      " << json_str(disasm(r.src[k])) << (k + 1 < r.src.size() ? ",\n" : "\n");
        os << "    ],\n    \"replacement\": [\n";
        for (size_t k = 0; k < r.rep.size(); k++)
            os << "      " << json_str(disasm(r.rep[k])) << (k + 1 < r.rep.size() ? ",\n" : "\n");
        os << "    ],\n    \"bytes_saved\": " << r.bytes_saved << ",\n    \"cycles_saved\": " << r.cycles_saved;
        std::string d = dead_desc(r.dead);
        if (!d.empty()) os << ",\n    \"dead_flags\": " << json_str(d);
        os << "\n  }" << (i + 1 < rules.size() ? ",\n" : "\n");
    }
    os << "]\n";
}

std::vector<uint16_t> decode_target(uint64_t id, int len, const uint16_t* tab) {
    std::vector<uint16_t> t((size_t)len);
    for (int k = len - 1; k >= 0; k--) { t[(size_t)k] = tab[id % 2863]; id /= 2863; }
    return t;
}

int cmd_enumerate(const Args& a) {
    uint8_t dead = 0;
    if (!parse_dead(a.get("--dead-flags", "none"), &dead)) {
        std::fprintf(stderr, "invalid --dead-flags value: use none, all, or hex (e.g. 0xFF)\n");
        return 1;
    }
    int max_target = (int)a.num("--max-target", 2);
    bool jsonl = a.has("--jsonl");
    std::string sem = a.get("--semantics", jsonl ? "cuda" : "go");
    bool go = sem == "go";
    std::string sweep = a.get("--sweep", go ? "reference" : "full");
    bool verbose = a.has("-v") || a.has("--verbose");
    uint32_t first = (uint32_t)a.num("--first-op-start", 0), last = (uint32_t)a.num("--first-op-end", 2863);
    if (max_target < 2 || max_target > 3) { std::fprintf(stderr, "--max-target must be 2 or 3\n"); return 1; }
    m6502_ctx* ctx = open_ctx((int)a.num("--gpu-id", 0));
    uint16_t tab[2863];
    m6502_insn_table(M6502_SEM_CUDA, tab);
    FILE* info = jsonl ? stderr : stdout;
    std::fprintf(info, "6502 Superoptimizer\n  Max target length: %d\n  Instructions: %d per position\n  Workers: %s\n",
                 max_target, 2863, a.get("--workers", "GPU").c_str());
    if (dead) std::fprintf(info, "  Dead flags: 0x%02X (%s)\n", dead, dead_desc(dead).c_str());
    std::fprintf(info, "\n");

    // Resume watermark: a checkpoint file holds "LEN NEXT", the target length
    // being enumerated and the next first-op index of it to run (every length
    // below LEN is complete).  The reference's only resume is the manual
    // --first-op-start (cuda/6502_search_v2.cu:776); its gob checkpoint is
    // never called (cmd/6502opt/main.go:74).
    std::string ckpt = a.get("--checkpoint", "");
    int resume_len = 2;
    uint32_t resume_at = first;
    if (!ckpt.empty()) {
        std::ifstream in(ckpt);
        int l;
        uint32_t w;
        if (in >> l >> w && l >= 2 && l <= max_target + 1) {
            resume_len = l;
            resume_at = std::max(first, std::min(w, last));
            std::fprintf(stderr, "resuming at target length %d, first-op %u\n", resume_len, resume_at);
        }
    }
    m6502_search_cfg cfg{};
    cfg.semantics = go ? M6502_SEM_GO : M6502_SEM_CUDA;
    cfg.sweep = sweep == "reference" ? M6502_SWEEP_REFERENCE : M6502_SWEEP_FULL;
    cfg.stages = a.has("--no-exhaust") ? (M6502_CHECK_QC | M6502_CHECK_MID) : M6502_CHECK_ALL;
    // The Go search tries candidates of length 1..max-target - 1 (search.go:26-28);
    // the CUDA pipeline only length 1 (6502_search_v2.cu:800-806).
    cfg.max_cand_len = go ? (uint32_t)max_target - 1 : 1;
    cfg.dead_flags = dead;
    std::vector<OutRule> all;
    uint64_t total_rules = 0;
    for (int len = resume_len; len <= max_target; len++) {
        if (verbose) std::fprintf(info, "=== Searching target length %d ===\n", len);
        const uint32_t start = len == resume_len ? resume_at : first;
        // Slices of first-op indices keep host buffers bounded and allow resume:
        // with --checkpoint the watermark advances every 64 first-ops.
        const uint32_t slice = len == 2 ? (ckpt.empty() ? 2863u : 64u) : 4u;
        for (uint32_t f = start; f < last; f += slice) {
            uint32_t f1 = std::min(last, f + slice);
            std::vector<m6502_rule> out(1u << 20);
            uint64_t n = 0;
            m6502_stats st{};
            int rc;
            while ((rc = m6502_enumerate(ctx, &cfg, (uint32_t)len, f, f1, out.data(), out.size(), &n, &st)) ==
                   M6502_E_OVERFLOW)
                out.resize(n);
            if (rc != M6502_OK) die(ctx, rc, "m6502_enumerate");
            total_rules += n;
            std::sort(out.begin(), out.begin() + (long)n, [](const m6502_rule& x, const m6502_rule& y) {
                if (x.target != y.target) return x.target < y.target;
                if (x.cand_len != y.cand_len) return x.cand_len < y.cand_len;
                return x.cand[0] != y.cand[0] ? x.cand[0] < y.cand[0] : x.cand[1] < y.cand[1];
            });
            for (uint64_t i = 0; i < n; i++) {
                const m6502_rule& r = out[i];
                std::vector<uint16_t> t = decode_target(r.target, len, tab);
                if (jsonl) {
                    char buf[512];
                    m6502_format_jsonl(t.data(), len, &r, dead, buf, sizeof buf);
                    std::fputs(buf, stdout);
                    std::fputc('\n', stdout);
                } else {
                    uint32_t semb = go ? M6502_SEM_GO : M6502_SEM_CUDA;
                    OutRule o{t, std::vector<uint16_t>(r.cand, r.cand + r.cand_len),
                              m6502_seq_bytes(t.data(), len, semb) - m6502_seq_bytes(r.cand, r.cand_len, semb),
                              m6502_seq_cycles(t.data(), len) - m6502_seq_cycles(r.cand, r.cand_len), r.dead_flags};
                    if (verbose)
                        std::printf("  FOUND%s: %s -> %s (-%d bytes, -%d cycles)\n",
                                    r.dead_flags ? (" (dead flags 0x" + std::string(1, "0123456789ABCDEF"[r.dead_flags >> 4]) +
                                                    std::string(1, "0123456789ABCDEF"[r.dead_flags & 15]) + ")").c_str() : "",
                                    disasm_seq(t.data(), len).c_str(), disasm_seq(r.cand, r.cand_len).c_str(),
                                    o.bytes_saved, o.cycles_saved);
                    all.push_back(std::move(o));
                }
            }
            if (jsonl) std::fflush(stdout);
            std::fprintf(stderr, "  [len %d] first-op %u..%u | targets:%llu | QC:%llu Mid:%llu Ex:%llu | found:%llu | %.0f ms\n",
                         len, f, f1, (unsigned long long)st.targets, (unsigned long long)st.qc_hits,
                         (unsigned long long)st.mid_hits, (unsigned long long)st.exh_checked,
                         (unsigned long long)n, st.ms_device);
            if (!ckpt.empty()) {   // written after the slice's rules are out
                std::ofstream o(ckpt);
                if (f1 < last) o << len << " " << f1 << "\n";
                else o << len + 1 << " " << first << "\n";
            }
        }
    }
    if (!jsonl) {
        std::stable_sort(all.begin(), all.end(), [](const OutRule& x, const OutRule& y) {
            return x.bytes_saved != y.bytes_saved ? x.bytes_saved > y.bytes_saved : x.cycles_saved > y.cycles_saved;
        });
        std::printf("\nFound %zu optimizations\n", all.size());
        std::string output = a.get("--output", "");
        if (!output.empty()) {
            std::ofstream os(output);
            if (!os) { std::fprintf(stderr, "cannot write %s\n", output.c_str()); return 1; }
            write_json(os, all);
            std::printf("Written to %s\n", output.c_str());
        }
    } else {
        std::fprintf(stderr, "Results found:      %llu\n", (unsigned long long)total_rules);
    }
    m6502_destroy(ctx);
    return 0;
}

int cmd_target(const Args& a) {
    if (a.pos.empty()) { std::fprintf(stderr, "usage: 6502opt target \"INSN : INSN ...\"\n"); return 1; }
    std::string input;
    for (size_t i = 0; i < a.pos.size(); i++) { if (i) input += " "; input += a.pos[i]; }
    uint16_t seq[16];
    int n = m6502_parse(input.c_str(), seq, 16);
    if (n < 0) { std::fprintf(stderr, "failed to parse: %s\n", input.c_str()); return 1; }
    if (n > 3) { std::fprintf(stderr, "targets of more than 3 instructions: use `6502opt stoke`\n"); return 1; }
    uint8_t dead = 0;
    if (!parse_dead(a.get("--dead-flags", "none"), &dead)) { std::fprintf(stderr, "invalid --dead-flags\n"); return 1; }
    // The Go CLI defaults to 4 (cmd/6502opt/main.go:130); the engine searches
    // candidates of length 1 and 2, so this command defaults to 2 and refuses
    // more rather than silently searching less than asked.
    long maxc = a.num("--max-candidate", 2);
    if (maxc > 2) {
        std::fprintf(stderr, "--max-candidate %ld: the GPU engine searches candidates of length 1..2\n", maxc);
        return 1;
    }
    std::printf("Target: %s (%d bytes, %d cycles)\n", input.c_str(), m6502_seq_bytes(seq, n, M6502_SEM_GO),
                m6502_seq_cycles(seq, n));
    m6502_ctx* ctx = open_ctx((int)a.num("--gpu-id", 0));
    m6502_search_cfg cfg{};
    cfg.semantics = M6502_SEM_GO;
    cfg.sweep = M6502_SWEEP_REFERENCE;
    cfg.max_cand_len = (uint32_t)std::max(0L, maxc);
    cfg.dead_flags = dead;
    m6502_rule out[4];
    uint64_t k = 0;
    int rc = maxc >= 1 ? m6502_search(ctx, &cfg, seq, 1, (uint32_t)n, out, 4, &k, nullptr) : M6502_OK;
    if (rc != M6502_OK) die(ctx, rc, "m6502_search");
    // SearchSingle(Masked) returns the best rule: most bytes, then cycles saved.
    int best = -1, bb = -1, bc = -1;
    for (uint64_t i = 0; i < k; i++) {
        int b = m6502_seq_bytes(seq, n, M6502_SEM_GO) - m6502_seq_bytes(out[i].cand, out[i].cand_len, M6502_SEM_GO);
        int c = m6502_seq_cycles(seq, n) - m6502_seq_cycles(out[i].cand, out[i].cand_len);
        if (b > bb || (b == bb && c > bc)) { best = (int)i; bb = b; bc = c; }
    }
    if (best < 0) std::printf("No shorter replacement found.\n");
    else std::printf("Replacement: %s (-%d bytes, -%d cycles)\n", disasm_seq(out[best].cand, out[best].cand_len).c_str(), bb, bc);
    m6502_destroy(ctx);
    return 0;
}

// Value of a string field in one JSON object line (no nesting needed here).
bool json_field(const std::string& line, const std::string& key, std::string* out) {
    std::string pat = "\"" + key + "\"";
    size_t p = line.find(pat);
    if (p == std::string::npos) return false;
    p = line.find(':', p + pat.size());
    if (p == std::string::npos) return false;
    p = line.find('"', p);
    if (p == std::string::npos) return false;
    std::string v;
    for (size_t i = p + 1; i < line.size(); i++) {
        if (line[i] == '\\' && i + 1 < line.size()) { v += line[++i]; continue; }
        if (line[i] == '"') { *out = v; return true; }
        v += line[i];
    }
    return false;
}

int cmd_verify(const Args& a) {
    if (a.pos.empty()) { std::fprintf(stderr, "usage: 6502opt verify-jsonl FILE\n"); return 1; }
    uint8_t dead = 0;
    if (!parse_dead(a.get("--dead-flags", "none"), &dead)) { std::fprintf(stderr, "invalid --dead-flags\n"); return 1; }
    bool verbose = a.has("-v") || a.has("--verbose");
    uint32_t sweep = a.get("--sweep", "reference") == "full" ? M6502_SWEEP_FULL : M6502_SWEEP_REFERENCE;
    std::ifstream in(a.pos[0]);
    if (!in) { std::fprintf(stderr, "cannot open %s\n", a.pos[0].c_str()); return 1; }
    m6502_ctx* ctx = open_ctx((int)a.num("--gpu-id", 0));
    // A rule whose sweep would exceed the engine's cone cap (bit 3 of
    // m6502_check_pairs) was not decided: it is reported as UNDECIDED, not as
    // a failure, and makes the command exit non-zero like a failure.
    uint64_t total = 0, passed = 0, failed = 0, skipped = 0, undecided = 0;
    std::vector<uint16_t> ti, ci;
    std::vector<uint32_t> to{0}, co{0};
    std::vector<std::pair<uint64_t, std::string>> names;
    auto flush = [&]() {
        size_t n = names.size();
        if (!n) return;
        std::vector<uint8_t> res(n);
        int rc = m6502_check_pairs(ctx, n, ti.data(), to.data(), ci.data(), co.data(), dead, M6502_CHECK_EXH, sweep,
                                   M6502_EXH_CONES, res.data(), nullptr);
        if (rc != M6502_OK) die(ctx, rc, "m6502_check_pairs");
        for (size_t i = 0; i < n; i++) {
            if (res[i] & M6502_CHECK_EXH) {
                passed++;
                if (verbose) std::printf("  [%llu] PASS: %s\n", (unsigned long long)names[i].first, names[i].second.c_str());
            } else if (res[i] & 8) {
                undecided++;
                std::printf("  [%llu] UNDECIDED: %s\n", (unsigned long long)names[i].first, names[i].second.c_str());
            } else {
                failed++;
                std::printf("  [%llu] FAIL: %s\n", (unsigned long long)names[i].first, names[i].second.c_str());
            }
        }
        ti.clear(); ci.clear(); to.assign(1, 0); co.assign(1, 0); names.clear();
    };
    std::string line;
    while (std::getline(in, line)) {
        size_t b = line.find_first_not_of(" \t\r\n");
        if (b == std::string::npos) continue;
        total++;
        std::string src, rep;
        uint16_t s[16], r[16];
        int ns, nr;
        if (!json_field(line, "source_asm", &src) || !json_field(line, "replacement_asm", &rep)) {
            std::fprintf(stderr, "  [%llu] JSON parse error\n", (unsigned long long)total);
            skipped++;
            continue;
        }
        if ((ns = m6502_parse(src.c_str(), s, 16)) < 0) {
            std::fprintf(stderr, "  [%llu] Cannot parse source \"%s\"\n", (unsigned long long)total, src.c_str());
            skipped++;
            continue;
        }
        if ((nr = m6502_parse(rep.c_str(), r, 16)) < 0) {
            std::fprintf(stderr, "  [%llu] Cannot parse replacement \"%s\"\n", (unsigned long long)total, rep.c_str());
            skipped++;
            continue;
        }
        ti.insert(ti.end(), s, s + ns);
        to.push_back((uint32_t)ti.size());
        ci.insert(ci.end(), r, r + nr);
        co.push_back((uint32_t)ci.size());
        names.emplace_back(total, src + " -> " + rep);
        if (names.size() >= (1u << 20)) flush();
    }
    flush();
    std::printf("\nVerification complete: %llu total, %llu passed, %llu failed, %llu skipped",
                (unsigned long long)total, (unsigned long long)passed, (unsigned long long)failed,
                (unsigned long long)skipped);
    if (undecided) std::printf(", %llu undecided", (unsigned long long)undecided);
    std::printf("\n");
    m6502_destroy(ctx);
    if (failed) {
        std::fprintf(stderr, "Error: %llu rules failed verification\n", (unsigned long long)failed);
        return 1;
    }
    if (undecided) {
        std::fprintf(stderr, "Error: %llu rules were not decided (sweep beyond the engine's cap)\n",
                     (unsigned long long)undecided);
        return 1;
    }
    return 0;
}

// stoke (cmd/6502opt/main.go:204-276): batched chains on the GPU, unique
// proven rewrites printed as stoke.Deduplicate (pkg/stoke/search.go:179-190)
// leaves them.
int cmd_stoke(const Args& a) {
    std::string target = a.get("--target", "");
    if (target.empty()) { std::fprintf(stderr, "--target is required\n"); return 1; }
    uint16_t seq[16];
    int n = m6502_parse(target.c_str(), seq, 16);
    if (n < 0 || n > 14) { std::fprintf(stderr, "failed to parse target: %s\n", target.c_str()); return 1; }
    uint8_t dead = 0;
    if (!parse_dead(a.get("--dead-flags", "none"), &dead)) { std::fprintf(stderr, "invalid --dead-flags\n"); return 1; }
    m6502_stoke_cfg cfg{};
    cfg.chains_per_target = (uint32_t)a.num("--chains", 128);
    cfg.steps = (uint64_t)a.num("--iterations", 10000000);
    cfg.steps_per_epoch = (uint32_t)a.num("--steps-per-epoch", 1000);
    cfg.decay = std::strtod(a.get("--decay", "0.9999").c_str(), nullptr);
    cfg.seed = (uint64_t)a.num("--seed", (long)std::chrono::steady_clock::now().time_since_epoch().count());
    cfg.cost = a.get("--cost", "ref") == "hamming" ? M6502_COST_HAMMING : M6502_COST_REF;
    cfg.sweep = a.get("--sweep", "reference") == "full" ? M6502_SWEEP_FULL : M6502_SWEEP_REFERENCE;
    cfg.dead_flags = dead;
    bool verbose = a.has("-v") || a.has("--verbose");
    uint32_t offs[2] = {0, (uint32_t)n};
    if (verbose)
        std::printf("STOKE search: %u chains x %llu iterations (decay=%.6f)\nTarget: %s (%d bytes, %d cycles)\n\n",
                    cfg.chains_per_target, (unsigned long long)cfg.steps, cfg.decay, disasm_seq(seq, n).c_str(),
                    m6502_seq_bytes(seq, n, M6502_SEM_GO), m6502_seq_cycles(seq, n));
    m6502_ctx* ctx = open_ctx((int)a.num("--gpu-id", 0));
    m6502_stoke_result res;
    std::vector<m6502_stoke_proof> proofs(1u << 16);
    uint64_t np = 0;
    m6502_stoke_stats st{};
    int rc;
    while ((rc = m6502_stoke_run(ctx, &cfg, seq, offs, 1, &res, proofs.data(), proofs.size(), &np, &st)) ==
           M6502_E_OVERFLOW)
        proofs.resize(np);
    if (rc != M6502_OK) die(ctx, rc, "m6502_stoke_run");
    // Deduplicate by replacement, keeping the first occurrence.
    std::vector<OutRule> uniq;
    std::vector<std::vector<uint16_t>> seen;
    for (uint64_t i = 0; i < np; i++) {
        std::vector<uint16_t> r(proofs[i].cand, proofs[i].cand + proofs[i].cand_len);
        if (std::find(seen.begin(), seen.end(), r) != seen.end()) continue;
        seen.push_back(r);
        if (verbose)
            std::printf("  Chain %u @ iter %llu: %s VERIFIED\n", proofs[i].chain, (unsigned long long)proofs[i].step,
                        disasm_seq(r.data(), (int)r.size()).c_str());
        uniq.push_back(OutRule{std::vector<uint16_t>(seq, seq + n), r,
                               m6502_seq_bytes(seq, n, M6502_SEM_GO) - m6502_seq_bytes(r.data(), (int)r.size(), M6502_SEM_GO),
                               m6502_seq_cycles(seq, n) - m6502_seq_cycles(r.data(), (int)r.size()), proofs[i].dead_flags});
    }
    if (verbose)
        std::printf("\nSTOKE complete: %llu verified results in %.0f ms\n", (unsigned long long)np, st.ms_device);
    std::printf("\n%zu unique optimizations found\n", uniq.size());
    for (size_t i = 0; i < uniq.size(); i++) {
        const OutRule& r = uniq[i];
        if (r.dead)
            std::printf("  %zu. %s (-%d bytes, -%d cycles, dead flags: %s)\n", i + 1,
                        disasm_seq(r.rep.data(), (int)r.rep.size()).c_str(), r.bytes_saved, r.cycles_saved,
                        dead_desc(r.dead).c_str());
        else
            std::printf("  %zu. %s (-%d bytes, -%d cycles)\n", i + 1, disasm_seq(r.rep.data(), (int)r.rep.size()).c_str(),
                        r.bytes_saved, r.cycles_saved);
    }
    std::string output = a.get("--output", "");
    if (!output.empty() && !uniq.empty()) {
        std::ofstream os(output);
        if (!os) { std::fprintf(stderr, "cannot write %s\n", output.c_str()); return 1; }
        write_json(os, uniq);
        std::printf("Written to %s\n", output.c_str());
    }
    m6502_destroy(ctx);
    return 0;
}

void usage() {
    std::fprintf(stderr,
                 "6502opt -- 6502 superoptimizer on the B200 engine\n\n"
                 "  enumerate      enumerate all target sequences and find shorter replacements\n"
                 "  target         find the optimal replacement for one instruction sequence\n"
                 "  verify-jsonl   verify JSONL rules with ExhaustiveCheck on the GPU\n"
                 "  stoke          STOKE stochastic search (batched MCMC chains on the GPU)\n"
                 "  export         export a rules JSON file as Go peephole code (-f go)\n");
}

// ---- export: the JSON rule array (WriteJSON's layout) -> Go peephole code ----

// Minimal reader of the JSON array that `enumerate --output` writes
// (pkg/result/output.go:21-35 layout): per object the string arrays
// "source" and "replacement" and the integers "bytes_saved",
// "cycles_saved"; other keys are skipped.
struct JsonRule {
    std::vector<std::string> source, replacement;
    long bytes_saved = 0, cycles_saved = 0;
};

struct JsonReader {
    const std::string& s;
    size_t i = 0;
    explicit JsonReader(const std::string& text) : s(text) {}
    void ws() { while (i < s.size() && std::isspace((unsigned char)s[i])) i++; }
    bool eat(char c) { ws(); if (i < s.size() && s[i] == c) { i++; return true; } return false; }
    bool str(std::string* out) {
        ws();
        if (i >= s.size() || s[i] != '"') return false;
        std::string r;
        for (i++; i < s.size() && s[i] != '"'; i++) {
            if (s[i] == '\\' && i + 1 < s.size()) i++;
            r += s[i];
        }
        if (i >= s.size()) return false;
        i++;
        *out = r;
        return true;
    }
    bool num(long* out) {
        ws();
        size_t j = i;
        if (j < s.size() && (s[j] == '-' || s[j] == '+')) j++;
        while (j < s.size() && std::isdigit((unsigned char)s[j])) j++;
        if (j == i) return false;
        *out = std::strtol(s.substr(i, j - i).c_str(), nullptr, 10);
        i = j;
        return true;
    }
    bool skip_value() {   // a value not needed: string, number, literal, array or object
        ws();
        std::string tmp;
        long n;
        if (i < s.size() && s[i] == '"') return str(&tmp);
        if (i < s.size() && (s[i] == '[' || s[i] == '{')) {
            const char open = s[i], close = open == '[' ? ']' : '}';
            i++;
            if (eat(close)) return true;
            do {
                if (open == '{' && !(str(&tmp) && eat(':'))) return false;
                if (!skip_value()) return false;
            } while (eat(','));
            return eat(close);
        }
        if (num(&n)) return true;
        for (const char* lit : {"true", "false", "null"})
            if (s.compare(i, std::strlen(lit), lit) == 0) { i += std::strlen(lit); return true; }
        return false;
    }
    bool str_array(std::vector<std::string>* out) {
        if (!eat('[')) return false;
        if (eat(']')) return true;
        do {
            std::string v;
            if (!str(&v)) return false;
            out->push_back(v);
        } while (eat(','));
        return eat(']');
    }
    bool rules(std::vector<JsonRule>* out) {
        if (!eat('[')) return false;
        if (eat(']')) return true;
        do {
            JsonRule r;
            if (!eat('{')) return false;
            if (!eat('}')) {
                do {
                    std::string key;
                    if (!str(&key) || !eat(':')) return false;
                    bool ok;
                    if (key == "source") ok = str_array(&r.source);
                    else if (key == "replacement") ok = str_array(&r.replacement);
                    else if (key == "bytes_saved") ok = num(&r.bytes_saved);
                    else if (key == "cycles_saved") ok = num(&r.cycles_saved);
                    else ok = skip_value();
                    if (!ok) return false;
                } while (eat(','));
                if (!eat('}')) return false;
            }
            out->push_back(r);
        } while (eat(','));
        return eat(']');
    }
};

// Go's %q of a disassembled instruction (printable ASCII: quote and backslash escaped).
std::string go_quote(const std::string& s) { return json_str(s); }

// export -f go (cmd/6502opt/main.go:147-194, WriteGoCode pkg/result/output.go:47-75).
// As in the reference, the JSON's dead_flags are not carried into the code.
int cmd_export(const Args& a) {
    if (a.pos.size() != 1) { std::fprintf(stderr, "usage: 6502opt export [-f go] rules.json\n"); return 1; }
    const std::string fmt = a.get("-f", a.get("--format", "go"));
    std::ifstream in(a.pos[0]);
    if (!in) { std::fprintf(stderr, "open %s: no such file\n", a.pos[0].c_str()); return 1; }
    std::string text((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    std::vector<JsonRule> jr;
    JsonReader rd(text);
    if (!rd.rules(&jr)) { std::fprintf(stderr, "invalid rules JSON: %s\n", a.pos[0].c_str()); return 1; }
    if (fmt != "go") { std::fprintf(stderr, "unknown format: %s\n", fmt.c_str()); return 1; }
    struct Parsed { std::vector<uint16_t> src, rep; long b, c; };
    std::vector<Parsed> rules;
    auto parse_slice = [](const std::vector<std::string>& v, std::vector<uint16_t>* out, std::string* bad) {
        for (const std::string& x : v) {
            uint16_t one[2];
            if (m6502_parse(x.c_str(), one, 2) != 1) { *bad = x; return false; }
            out->push_back(one[0]);
        }
        return true;
    };
    for (const JsonRule& r : jr) {
        Parsed p{{}, {}, r.bytes_saved, r.cycles_saved};
        std::string bad;
        if (!parse_slice(r.source, &p.src, &bad)) {
            std::fprintf(stderr, "skipping rule (bad source): %s\n", bad.c_str());
            continue;
        }
        if (!parse_slice(r.replacement, &p.rep, &bad)) {
            std::fprintf(stderr, "skipping rule (bad replacement): %s\n", bad.c_str());
            continue;
        }
        rules.push_back(p);
    }
    auto join = [](const std::vector<uint16_t>& v) {
        std::string s;
        for (size_t k = 0; k < v.size(); k++) { if (k) s += " : "; s += disasm(v[k]); }
        return s;
    };
    auto slice = [](const std::vector<uint16_t>& v) {
        std::string s = "[]string{";
        for (size_t k = 0; k < v.size(); k++) { if (k) s += ", "; s += go_quote(disasm(v[k])); }
        return s + "}";
    };
    std::printf("package peephole\n\n// Generated by 6502opt. DO NOT EDIT.\n\n");
    std::printf("type PeepholeRule struct {\n\tSource      []string\n\tReplacement []string\n"
                "\tBytesSaved  int\n\tCyclesSaved int\n\tDeadFlags   string\n}\n\n");
    std::printf("var Rules = []PeepholeRule{\n");
    for (const Parsed& p : rules) {
        std::printf("\t// %s -> %s (-%ld bytes, -%ld cycles)\n", join(p.src).c_str(), join(p.rep).c_str(), p.b, p.c);
        std::printf("\t{Source: %s, Replacement: %s, BytesSaved: %ld, CyclesSaved: %ld},\n", slice(p.src).c_str(),
                    slice(p.rep).c_str(), p.b, p.c);
    }
    std::printf("}\n");
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) { usage(); return 1; }
    std::string cmd = argv[1];
    Args a = parse_args(argc, argv, 2);
    if (cmd == "enumerate") return cmd_enumerate(a);
    if (cmd == "target") return cmd_target(a);
    if (cmd == "verify-jsonl") return cmd_verify(a);
    if (cmd == "stoke") return cmd_stoke(a);
    if (cmd == "export") return cmd_export(a);
    usage();
    return 1;
}
