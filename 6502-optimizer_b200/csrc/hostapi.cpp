// hostapi.cpp -- host-only helpers of the C ABI: instruction tables,
// disassembly, assembly parsing, pruning, byte/cycle counts, the dataflow
// model and the JSONL formatter.  Compiled into libm6502gpu.so beside the
// kernels; none of these touch the GPU.
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>

#include "isa.cuh"
#include "m6502.h"

using namespace m6502;

namespace {

// Mnemonics in opcode order (pkg/inst/catalog.go:105-201); immediates get
// " #$XX" appended.
const char* const kMnemonic[NUM_OPS] = {
    "TAX", "TAY", "TXA", "TYA", "TSX", "TXS", "INX", "INY", "DEX", "DEY",
    "ASL A", "LSR A", "ROL A", "ROR A",
    "CLC", "SEC", "CLD", "SED", "CLI", "SEI", "CLV",
    "PHA", "PLA", "PHP", "PLP", "NOP",
    "LDA", "LDX", "LDY", "ADC", "SBC", "AND", "ORA", "EOR", "CMP", "CPX", "CPY",
    "LDA M", "LDX M", "LDY M", "STA M", "STX M", "STY M", "ADC M", "SBC M",
    "AND M", "ORA M", "EOR M", "CMP M", "CPX M", "CPY M", "INC M", "DEC M",
    "ASL M", "LSR M", "ROL M", "ROR M", "BIT M"};

const char kHex[] = "0123456789ABCDEF";

// Appenders of the JSONL writer: each writes at q and returns the new end.
char* put_str(char* q, const char* s) {
    while (*s) *q++ = *s++;
    return q;
}
// The disassembly of a valid instruction, as m6502_disasm prints it.
char* put_insn(char* q, uint16_t insn) {
    const uint32_t op = insn & 0xFFu;
    q = put_str(q, kMnemonic[op]);
    if (has_imm(op)) {
        const uint32_t v = insn >> 8;
        *q++ = ' '; *q++ = '#'; *q++ = '$'; *q++ = kHex[v >> 4]; *q++ = kHex[v & 15];
    }
    return q;
}
char* put_int(char* q, int v) {
    unsigned u = v < 0 ? 0u - (unsigned)v : (unsigned)v;
    if (v < 0) *q++ = '-';
    char d[10];
    int k = 0;
    do { d[k++] = (char)('0' + u % 10); u /= 10; } while (u);
    while (k) *q++ = d[--k];
    return q;
}

std::string trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && std::isspace((unsigned char)s[a])) a++;
    while (b > a && std::isspace((unsigned char)s[b - 1])) b--;
    return s.substr(a, b - a);
}

// parseImmediate (cmd/6502opt/main.go:467-494): $FF, 0xFF, FFH or decimal.
bool parse_imm(std::string s, unsigned* v) {
    s = trim(s);
    if (s.empty()) return false;
    int base = 10;
    if (s[0] == '$') { s = s.substr(1); base = 16; }
    else if (s.size() > 2 && s[0] == '0' && (s[1] == 'x' || s[1] == 'X')) { s = s.substr(2); base = 16; }
    else if (std::toupper((unsigned char)s.back()) == 'H') { s.pop_back(); base = 16; }
    if (s.empty()) return false;
    char* end = nullptr;
    unsigned long x = std::strtoul(s.c_str(), &end, base);
    if (!end || *end || x > 0xFFFF) return false;
    *v = (unsigned)x;
    return true;
}

// parseSingleInstruction (cmd/6502opt/main.go:337-384).
bool parse_one(const std::string& text, uint16_t* out) {
    std::string up = trim(text);
    for (auto& ch : up) ch = (char)std::toupper((unsigned char)ch);
    for (uint32_t op = 0; op < NUM_OPS; op++) {
        if (!has_imm(op)) {
            if (up == kMnemonic[op]) { *out = (uint16_t)op; return true; }
            continue;
        }
        std::string prefix = std::string(kMnemonic[op]) + " #";
        if (up.compare(0, prefix.size(), prefix) != 0) continue;
        unsigned v;
        if (!parse_imm(up.substr(prefix.size()), &v)) continue;
        *out = (uint16_t)(op | ((v & 0xFFu) << 8));
        return true;
    }
    return false;
}

bool valid(const uint16_t* s, int n) {
    for (int i = 0; i < n; i++) if ((s[i] & 0xFF) >= NUM_OPS) return false;
    return true;
}

}  // namespace

extern "C" {

int m6502_insn_table(uint32_t semantics, uint16_t* out) {
    if (!out || semantics > M6502_SEM_GO) return M6502_E_INVAL;
    int k = 0;
    if (semantics == M6502_SEM_GO) {
        for (uint32_t op = 0; op < NUM_OPS; op++) if (!has_imm(op)) out[k++] = (uint16_t)op;
        for (uint32_t op = 0; op < NUM_OPS; op++)
            if (has_imm(op)) for (uint32_t v = 0; v < 256; v++) out[k++] = (uint16_t)(op | (v << 8));
    } else {
        for (uint32_t op = 0; op < NUM_OPS; op++) {
            if (has_imm(op)) for (uint32_t v = 0; v < 256; v++) out[k++] = (uint16_t)(op | (v << 8));
            else out[k++] = (uint16_t)op;
        }
    }
    return k;
}

int m6502_disasm(uint16_t insn, char* buf, int cap) {
    if (!buf || cap <= 0) return M6502_E_INVAL;
    uint32_t op = insn & 0xFF;
    if (op >= NUM_OPS) return std::snprintf(buf, (size_t)cap, "OP(%u)", op);
    if (has_imm(op)) return std::snprintf(buf, (size_t)cap, "%s #$%02X", kMnemonic[op], insn >> 8);
    return std::snprintf(buf, (size_t)cap, "%s", kMnemonic[op]);
}

int m6502_parse(const char* text, uint16_t* out, int cap) {
    if (!text || !out || cap <= 0) return M6502_E_INVAL;
    std::string s(text);
    int n = 0;
    size_t pos = 0;
    while (pos <= s.size()) {
        size_t colon = s.find(':', pos);
        std::string part = trim(s.substr(pos, colon == std::string::npos ? std::string::npos : colon - pos));
        if (!part.empty()) {
            if (n >= cap) return M6502_E_INVAL;
            if (!parse_one(part, &out[n])) return M6502_E_INVAL;
            n++;
        }
        if (colon == std::string::npos) break;
        pos = colon + 1;
    }
    return n > 0 ? n : M6502_E_INVAL;
}

int m6502_should_prune(const uint16_t* seq, int n) {
    if (!seq || n < 0 || !valid(seq, n)) return M6502_E_INVAL;
    return should_prune(seq, n) ? 1 : 0;
}

int m6502_seq_bytes(const uint16_t* seq, int n, uint32_t semantics) {
    if (!seq || n < 0 || !valid(seq, n)) return M6502_E_INVAL;
    int b = 0;
    for (int i = 0; i < n; i++)
        b += (int)(semantics == M6502_SEM_GO ? bytes_go(seq[i] & 0xFF) : bytes_cuda(seq[i] & 0xFF));
    return b;
}

int m6502_seq_cycles(const uint16_t* seq, int n) {
    if (!seq || n < 0 || !valid(seq, n)) return M6502_E_INVAL;
    int c = 0;
    for (int i = 0; i < n; i++) c += (int)cycles(seq[i] & 0xFF);
    return c;
}

uint64_t m6502_enumerate_targets(uint32_t tlen, uint32_t first, uint32_t last, uint16_t* out, uint64_t cap) {
    if (tlen < 1 || tlen > 3) return 0;
    uint16_t tab[kNumInsns];
    m6502_insn_table(M6502_SEM_CUDA, tab);
    if (last > (uint32_t)kNumInsns) last = kNumInsns;
    uint64_t inner = 1;
    for (uint32_t i = 1; i < tlen; i++) inner *= (uint64_t)kNumInsns;
    uint64_t n = 0;
    uint16_t s[3];
    for (uint32_t f = first; f < last; f++) {
        s[0] = tab[f];
        for (uint64_t r = 0; r < inner; r++) {
            if (tlen == 2) s[1] = tab[r];
            if (tlen == 3) { s[1] = tab[r / kNumInsns]; s[2] = tab[r % kNumInsns]; }
            if (should_prune(s, (int)tlen)) continue;
            if (out && n < cap) std::memcpy(out + n * tlen, s, tlen * sizeof(uint16_t));
            n++;
        }
    }
    return n;
}

namespace {
// splitmix64 (Steele, Lea & Flood 2014).
uint64_t splitmix64(uint64_t* x) {
    uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
// Uniform index in [0, bound): rejection of the top partial block of 2^64.
uint32_t uniform_index(uint64_t* x, uint32_t bound) {
    uint64_t rem = (UINT64_MAX % bound + 1) % bound;
    uint64_t lim = rem ? UINT64_MAX - rem + 1 : 0;
    for (;;) {
        uint64_t r = splitmix64(x);
        if (lim == 0 || r < lim) return (uint32_t)(r % bound);
    }
}
}  // namespace

int m6502_draw_targets(uint64_t seed, uint32_t min_len, uint32_t max_len, uint64_t n, int reject_pruned,
                       uint16_t* insns, uint32_t* offs) {
    if (min_len < 1 || max_len < min_len || max_len > 16 || !insns || !offs) return M6502_E_INVAL;
    uint16_t tab[kNumInsns];
    m6502_insn_table(M6502_SEM_CUDA, tab);
    uint64_t x = seed, k = 0;
    offs[0] = 0;
    for (uint64_t i = 0; i < n;) {
        uint32_t len = min_len == max_len ? min_len : min_len + uniform_index(&x, max_len - min_len + 1);
        uint16_t s[16];
        for (uint32_t p = 0; p < len; p++) s[p] = tab[uniform_index(&x, kNumInsns)];
        if (reject_pruned && should_prune(s, (int)len)) continue;
        std::memcpy(insns + k, s, len * sizeof(uint16_t));
        k += len;
        offs[++i] = (uint32_t)k;
    }
    return M6502_OK;
}

int m6502_op_deps(int op, uint16_t deps[13]) {
    if (op < 0 || op >= (int)NUM_OPS || !deps) return M6502_E_INVAL;
    return (int)op_deps((uint32_t)op, deps);
}

int m6502_format_jsonl(const uint16_t* target, int tlen, const m6502_rule* rule, uint8_t run_dead_flags,
                       char* buf, int cap) {
    if (!target || !rule || !buf || cap <= 0 || tlen < 1 || rule->cand_len < 1 || rule->cand_len > 3 ||
        !valid(target, tlen) || !valid(rule->cand, rule->cand_len))
        return M6502_E_INVAL;
    // Written straight into a local line (an instruction is at most 10
    // characters, its separator 3), then copied like snprintf: at most cap - 1
    // characters and a NUL; the return value is the whole line's length.
    char local[1024];
    std::unique_ptr<char[]> heap;
    const size_t need = 256 + 13 * (size_t)(tlen + rule->cand_len);
    char* line = local;
    if (need > sizeof local) { heap.reset(new char[need]); line = heap.get(); }
    char* q = line;
    int sb = 0, cb = 0, cs = 0;
    q = put_str(q, "{\"source_asm\":\"");
    for (int i = 0; i < tlen; i++) {
        if (i) q = put_str(q, " : ");
        q = put_insn(q, target[i]);
        sb += (int)bytes_cuda(target[i] & 0xFF);
        cs += (int)cycles(target[i] & 0xFF);
    }
    q = put_str(q, "\",\"replacement_asm\":\"");
    for (int i = 0; i < rule->cand_len; i++) {
        if (i) q = put_str(q, " : ");
        q = put_insn(q, rule->cand[i]);
        cb += (int)bytes_cuda(rule->cand[i] & 0xFF);
        cs -= (int)cycles(rule->cand[i] & 0xFF);
    }
    q = put_str(q, "\",\"source_bytes\":");
    q = put_int(q, sb);
    q = put_str(q, ",\"replacement_bytes\":");
    q = put_int(q, cb);
    q = put_str(q, ",\"bytes_saved\":");
    q = put_int(q, sb - cb);
    q = put_str(q, ",\"cycles_saved\":");
    q = put_int(q, cs);
    if (run_dead_flags) {
        q = put_str(q, ",\"dead_flags\":\"0x");
        *q++ = kHex[run_dead_flags >> 4];
        *q++ = kHex[run_dead_flags & 15];
        *q++ = '"';
    }
    *q++ = '}';
    const int n = (int)(q - line);
    const int k = n < cap ? n : cap - 1;
    std::memcpy(buf, line, (size_t)k);
    buf[k] = '\0';
    return n;
}

}  // extern "C"
