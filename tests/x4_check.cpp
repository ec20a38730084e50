// Checks the four-states-per-register executors (exec_x4, and exec_x4d
// driven by the per-opcode descriptors of x4_desc) against four scalar exec
// calls for every instruction of the table on seeded random states.  Built and run by tests/test_abi_host.py::test_swar_exec_matches_scalar.
#include <cstdio>
#include <cstdint>

#include "isa.cuh"

using namespace m6502;

static uint64_t rng = 0x6502;
static uint32_t next8() {
    uint64_t z = (rng += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return (uint32_t)((z ^ (z >> 31)) & 0xFFu);
}

int main() {
    long checked = 0, bad = 0;
    for (uint32_t op = 0; op < NUM_OPS; op++) {
        for (uint32_t imm = 0; imm < (has_imm(op) ? 256u : 1u); imm++) {
            const uint32_t insn = op | (imm << 8);
            for (int trial = 0; trial < 64; trial++) {
                St one[4], packed{}, packed_d{};
                for (int k = 0; k < 4; k++) {
                    one[k] = {next8(), next8(), next8(), next8(), next8(), next8(), next8(), next8()};
                    if (trial < 8) one[k].a = (trial * 4 + k) & 1 ? 0u : 0x80u;   // zero / sign edge cases
                    uint32_t* f = &one[k].a;
                    uint32_t* g = &packed.a;
                    for (int i = 0; i < 8; i++) g[i] |= f[i] << (8 * k);
                }
                packed_d = packed;
                exec_x4(packed, insn);
                exec_x4d(packed_d, insn, x4_desc(op));
                for (int k = 0; k < 4; k++) {
                    exec(one[k], insn);
                    const uint32_t* f = &one[k].a;
                    const uint32_t* g = &packed.a;
                    const uint32_t* gd = &packed_d.a;
                    for (int i = 0; i < 8; i++) {
                        if (((g[i] >> (8 * k)) & 0xFFu) != (f[i] & 0xFFu) ||
                            ((gd[i] >> (8 * k)) & 0xFFu) != (f[i] & 0xFFu)) {
                            if (bad < 10) std::printf("mismatch op %u imm %u state %d field %d\n", op, imm, k, i);
                            bad++;
                        }
                    }
                }
                checked++;
            }
        }
    }
    std::printf("checked %ld packed executions, %ld mismatches\n", checked, bad);
    return bad ? 1 : 0;
}
