/* Prints the layout of every public struct of include/m6502.h, one line per
 * field: "<struct> <field> <offset> <size>", then "<struct> SIZEOF <size>".
 * Built and run by tests/test_abi_host.py::test_ctypes_layouts_match_the_header,
 * which compares it with the ctypes mirror in m6502/_lib.py. */
#include <stddef.h>
#include <stdio.h>

#include "m6502.h"

#define F(T, f) printf("%s %s %zu %zu\n", #T, #f, offsetof(T, f), sizeof(((T *)0)->f))
#define S(T) printf("%s SIZEOF %zu\n", #T, sizeof(T))

int main(void) {
    F(m6502_opts, device); F(m6502_opts, flags); F(m6502_opts, targets_per_pass); S(m6502_opts);

    F(m6502_rule, target); F(m6502_rule, cand); F(m6502_rule, cand_len); F(m6502_rule, dead_flags);
    S(m6502_rule);

    F(m6502_search_cfg, semantics); F(m6502_search_cfg, sweep); F(m6502_search_cfg, exh_mode);
    F(m6502_search_cfg, stages); F(m6502_search_cfg, max_cand_len); F(m6502_search_cfg, flags);
    F(m6502_search_cfg, dead_flags); F(m6502_search_cfg, reserved); S(m6502_search_cfg);

    F(m6502_stats, targets); F(m6502_stats, pairs); F(m6502_stats, qc_hits); F(m6502_stats, mid_hits);
    F(m6502_stats, exh_checked); F(m6502_stats, exh_passed); F(m6502_stats, rules); F(m6502_stats, exh_states);
    F(m6502_stats, exh_items); F(m6502_stats, exh_algo_ops); F(m6502_stats, passes);
    F(m6502_stats, exh_probe_rejects); F(m6502_stats, ms_device); F(m6502_stats, ms_fingerprint);
    F(m6502_stats, ms_qc); F(m6502_stats, ms_exhaustive); F(m6502_stats, ms_exh_items); F(m6502_stats, ms_emit);
    F(m6502_stats, graph_replays); F(m6502_stats, exh_undecided); S(m6502_stats);

    F(m6502_tune, exh_minb); F(m6502_tune, ticket_batch); F(m6502_tune, chunk_log2); F(m6502_tune, join_probe);
    F(m6502_tune, reserved); S(m6502_tune);

    F(m6502_stoke_cfg, chains_per_target); F(m6502_stoke_cfg, steps_per_epoch); F(m6502_stoke_cfg, steps);
    F(m6502_stoke_cfg, seed); F(m6502_stoke_cfg, decay); F(m6502_stoke_cfg, t_start); F(m6502_stoke_cfg, t_end);
    F(m6502_stoke_cfg, cost); F(m6502_stoke_cfg, max_len); F(m6502_stoke_cfg, sweep);
    F(m6502_stoke_cfg, stop_on_proof); F(m6502_stoke_cfg, proposal); F(m6502_stoke_cfg, dead_flags);
    F(m6502_stoke_cfg, uniform_chains); F(m6502_stoke_cfg, reserved); F(m6502_stoke_cfg, learned_frac);
    F(m6502_stoke_cfg, first_epoch); F(m6502_stoke_cfg, model); F(m6502_stoke_cfg, trajectories);
    F(m6502_stoke_cfg, traj_cap); F(m6502_stoke_cfg, traj_count); S(m6502_stoke_cfg);

    F(m6502_stoke_proof, target); F(m6502_stoke_proof, chain); F(m6502_stoke_proof, step);
    F(m6502_stoke_proof, ms); F(m6502_stoke_proof, cand); F(m6502_stoke_proof, cand_len);
    F(m6502_stoke_proof, dead_flags); F(m6502_stoke_proof, reserved); S(m6502_stoke_proof);

    F(m6502_stoke_result, first_proof_ms); F(m6502_stoke_result, first_proof_step); F(m6502_stoke_result, proofs);
    F(m6502_stoke_result, bytes_saved); F(m6502_stoke_result, cycles_saved); F(m6502_stoke_result, best);
    F(m6502_stoke_result, best_len); F(m6502_stoke_result, dead_flags); F(m6502_stoke_result, reserved);
    S(m6502_stoke_result);

    F(m6502_stoke_stats, steps); F(m6502_stoke_stats, accepted); F(m6502_stoke_stats, candidates);
    F(m6502_stoke_stats, proofs); F(m6502_stoke_stats, undecided); F(m6502_stoke_stats, epochs);
    F(m6502_stoke_stats, targets_proven); F(m6502_stoke_stats, ms_device); F(m6502_stoke_stats, ms_chains);
    F(m6502_stoke_stats, ms_verify); F(m6502_stoke_stats, verified); S(m6502_stoke_stats);

    F(m6502_mlp_example, target); F(m6502_mlp_example, cand); F(m6502_mlp_example, diff);
    F(m6502_mlp_example, tlen); F(m6502_mlp_example, clen); F(m6502_mlp_example, pos); F(m6502_mlp_example, op);
    F(m6502_mlp_example, imm); F(m6502_mlp_example, weight); F(m6502_mlp_example, reserved);
    S(m6502_mlp_example);
    return 0;
}
