/*
 * oracle/args_harness.c -- the reference's command-line parser alone
 * (GetCMLArgs, Solver/src/utils.c:34-460), for checking bin/ns2d's grammar.
 * Test infrastructure only.  Defines the globals main.c defines
 * (Solver/src/main.c:26-29), parses argv with the reference's own function
 * and prints the result in the key order of `ns2d --dry-run`; an invalid
 * argument ends the process in GetCMLArgs with the reference's exit(1).
 */
#include <stdio.h>
#include <stdlib.h>
#include "data_types.h"
#include "utils.h"

runtime_data_struct* run_data;
system_vars_struct* sys_vars;
HDF_file_info_struct* file_info;
stats_data_struct* stats_data;

int main(int argc, char** argv) {
    sys_vars = (system_vars_struct*)calloc(1, sizeof(system_vars_struct));
    run_data = (runtime_data_struct*)calloc(1, sizeof(runtime_data_struct));
    file_info = (HDF_file_info_struct*)calloc(1, sizeof(HDF_file_info_struct));
    stats_data = (stats_data_struct*)calloc(1, sizeof(stats_data_struct));
    GetCMLArgs(argc, argv);
    const system_vars_struct* s = sys_vars;
    printf("{\"N\": [%ld, %ld], \"t0\": %.17g, \"T\": %.17g, \"dt\": %.17g, \"adapt_step\": %d, \"cfl_cond\": %d, "
           "\"cfl_const\": %.17g, \"u0\": \"%s\", \"forcing\": \"%s\", \"force_k\": %d, \"force_scale\": %.17g, "
           "\"trans_iters\": %d, \"trans_frac\": %.17g, \"nu\": %.17g, \"hyper_flag\": %d, \"hyper_pow\": %.17g, "
           "\"ekmn_alpha\": %.17g, \"ekmn_flag\": %d, \"ekmn_pow\": %.17g, \"save_every\": %d, \"output_dir\": \"%s\", "
           "\"output_tag\": \"%s\", \"input_file\": \"%s\", \"file_only\": %d}\n",
           s->N[0], s->N[1], s->t0, s->T, s->dt, (int)s->ADAPT_STEP_FLAG, (int)s->CFL_COND_FLAG, s->CFL_CONST, s->u0,
           s->forcing, (int)s->force_k, s->force_scale_var, (int)s->TRANS_ITERS_FLAG, s->TRANS_ITERS_FRAC, s->NU,
           (int)s->HYPER_VISC_FLAG, (double)s->HYPER_VISC_POW, s->EKMN_ALPHA, (int)s->EKMN_DRAG_FLAG,
           (double)s->EKMN_DRAG_POW, (int)s->SAVE_EVERY, file_info->output_dir, file_info->output_tag,
           file_info->input_file_name, (int)file_info->file_only);
    return 0;
}
