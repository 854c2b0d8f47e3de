/*
 * args.c -- the reference's command-line grammar (GetCMLArgs,
 * Solver/src/utils.c:34-460) for bin/ns2d.
 *
 * Short options as the reference's getopt string "o:h:n:d:s:e:t:v:i:c:p:f:z:T:".
 * Several flags take their meaning from how often they have appeared:
 *   -o  1st: output directory, later: file-only output
 *   -n  1st: Nx, 2nd: Ny
 *   -h  1st: dt (> 0), later: adaptive-step flag (0/1)
 *   -c  1st: CFL-condition flag (0/1), later: CFL constant (> 0)
 *   -v  1st: viscosity (>= 0), 2nd: hyperviscosity flag (0/1), later: its power (> 0)
 *   -d  1st: Ekman drag (>= 0), 2nd: drag flag (0/1), later: drag power (<= 0)
 *   -f  1st: forcing name (a known one; others are ignored), 2nd: force_k, later: scale
 *   -T  1st: transient-iterations flag (0/1), later: fraction in (0, 1)
 *   -s  start time (>= 0), -e end time (>= 0, >= start), -p save every, -t tag,
 *   -i  initial condition (unknown names become "NONE"), -z input file (must exist).
 * An invalid value prints a diagnostic and exits with status 1, as the
 * reference does; where the reference would go on with a value that breaks it
 * later (a third -n, -p 0) this parser stops with status 1 as well.  Long
 * options select what the reference fixes when it is compiled:
 * --integrator=RK4CN|RK4|AB4|DP5, --dealias=23|HOU_LI, --precision=FP64|FP32,
 * --device=N, --no-quirks (corrected forms of the reference's quirks),
 * --phase-only (the -D__PHASE_ONLY model, RK4CN / RK4 only),
 * --dry-run (print the parameters as JSON and exit), --quiet.
 */
#include <getopt.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "run.h"

static void die_num(const char* fmt, double v) {
    fprintf(stderr, "\n[ERROR] Parsing of Command Line Arguments Failed: ");
    fprintf(stderr, fmt, v);
    fprintf(stderr, "\n-->> Exiting!\n\n");
    exit(1);
}
static void die_str(const char* fmt, const char* v) {
    fprintf(stderr, "\n[ERROR] Parsing of Command Line Arguments Failed: ");
    fprintf(stderr, fmt, v);
    fprintf(stderr, "\n-->> Exiting!\n\n");
    exit(1);
}

static void usage_and_exit(void) {
    fprintf(stderr,
            "\n[ERROR] Incorrect command line flag encountered\n"
            "Use -o to specify the output directory\n"
            "Use -n to specify the size of each dimension in the system\n"
            "Use -s to specify the start time of the simulation\n"
            "Use -e to specify the end time of the simulation\n"
            "Use -h to specify the timestep\n"
            "Use -c to specify the CFL constant for the adaptive stepping\n"
            "Use -v to specify the system viscosity\n"
            "Use -i to specify the initial condition\n"
            "Use -t to specify the tag name to be used in the output file directory\n"
            "Use -f to specify the forcing type\n"
            "Use -T to specify if transient iterations are to be performed\n"
            "Use -p to specify how often to print to file\n"
            "Use -z to specify an input file to read parameters from\n"
            "Long options: --integrator=RK4CN|RK4|AB4|DP5 --dealias=23|HOU_LI --precision=FP64|FP32\n"
            "              --device=N --no-quirks --phase-only --dry-run --quiet\n"
            "\nExample usage:\n\tns2d -o ../Data/Tmp/ -n 64 -n 64 -s 0.0 -e 1.0 -h 0.0001 -v 1.0 -i TG_VORT -t TEMP_RUN\n"
            "-->> Now Exiting!\n\n");
    exit(1);
}

static void copy(char* dst, size_t cap, const char* src) {
    strncpy(dst, src, cap - 1);
    dst[cap - 1] = '\0';
}

static int flag01(const char* arg, const char* what) {
    const int v = atoi(arg);
    if (v != 0 && v != 1) {
        fprintf(stderr, "\n[ERROR] Parsing of Command Line Arguments Failed: Incorrect %s flag: [%d] Must be either 0 or 1\n-->> Exiting!\n\n",
                what, v);
        exit(1);
    }
    return v;
}

/* Initial-condition names the reference accepts (utils.c:258-331). */
static const char* const k_initial[] = {"TG_VEL",           "TG_VORT",   "DOUBLE_SHEAR_LAYER", "TESTING",
                                        "DECAY_TURB_BB",    "DECAY_TURB_NB", "DECAY_TURB_ALT", "DECAY_TURB_EXP",
                                        "GAUSS_DECAY_TURB", "EXTRM_ENS", "MAX_PALIN",          "RING",
                                        "UNIF",             "RANDOM",    "GAUSS_BLOB",         "ZERO",
                                        "ZERO_KOLM",        NULL};
/* Forcing names (utils.c:383-411). */
static const char* const k_forcing[] = {"ZERO", "CONST_GAUSS", "KOLM", "STOC", "STOC_GAUSS", "NONE", NULL};

static int in_list(const char* s, const char* const* list) {
    for (int i = 0; list[i]; ++i)
        if (!strcmp(s, list[i])) return 1;
    return 0;
}

static void defaults(ns2d_run* r) {
    memset(r, 0, sizeof(*r));
    copy(r->input_file, sizeof(r->input_file), "NONE");
    copy(r->input_dir, sizeof(r->input_dir), "./Data/Solver/InitialConditions/");
    copy(r->output_dir, sizeof(r->output_dir), "./Data/Tmp/");
    copy(r->output_tag, sizeof(r->output_tag), "No-Tag");
    r->N[0] = r->N[1] = 64;
    r->t0 = 0.0;
    r->dt = 1e-4;
    r->T = 1.0;
    r->cfl_const = 0.9;
    r->adapt_step = 0;
    r->cfl_cond = 1;
    copy(r->u0, sizeof(r->u0), "TG_VORT");
    copy(r->forcing, sizeof(r->forcing), "NONE");
    r->force_k = 0;
    r->force_scale = 1.0;
    r->trans_iters = 0;
    r->trans_frac = 0.2;
    r->nu = 0.0001;
    r->hyper_flag = 0;
    r->hyper_pow = 2.0;
    r->ekmn_alpha = 0.0;
    r->ekmn_flag = 0;
    r->ekmn_pow = -2.0;
    r->save_every = 100;
    r->integrator = NS2D_RK4CN;
    r->dealias = NS2D_DEALIAS_23;
    r->precision = NS2D_FP64;
    r->device = 0;
    r->quirks = NS2D_QUIRKS_REFERENCE;
}

enum { OPT_INTEGRATOR = 1000, OPT_DEALIAS, OPT_PRECISION, OPT_DEVICE, OPT_NO_QUIRKS, OPT_DRY_RUN, OPT_QUIET,
       OPT_PHASE_ONLY };

void ns2d_cli_parse(int argc, char** argv, ns2d_run* r) {
    static const struct option longs[] = {{"integrator", required_argument, 0, OPT_INTEGRATOR},
                                          {"dealias", required_argument, 0, OPT_DEALIAS},
                                          {"precision", required_argument, 0, OPT_PRECISION},
                                          {"device", required_argument, 0, OPT_DEVICE},
                                          {"no-quirks", no_argument, 0, OPT_NO_QUIRKS},
                                          {"dry-run", no_argument, 0, OPT_DRY_RUN},
                                          {"quiet", no_argument, 0, OPT_QUIET},
                                          {"phase-only", no_argument, 0, OPT_PHASE_ONLY},
                                          {0, 0, 0, 0}};
    defaults(r);
    int seen_o = 0, seen_n = 0, seen_h = 0, seen_c = 0, seen_v = 0, seen_d = 0, seen_f = 0, seen_T = 0;
    int c;
    optind = 1;
    while ((c = getopt_long(argc, argv, "o:h:n:d:s:e:t:v:i:c:p:f:z:T:", longs, NULL)) != -1) {
        switch (c) {
            case 'o':
                if (seen_o++ == 0)
                    copy(r->output_dir, sizeof(r->output_dir), optarg);
                else
                    r->file_only = 1;
                break;
            case 'n': {
                if (seen_n >= 2) die_str("more than two -n dimensions given%s", "");
                const long v = atoi(optarg);
                if (v <= 2) die_num("The minimum dimension size of [%g] must be greater than 2", (double)v);
                if (v % 2 != 0) die_num("The system dimension of [%g] must be a multiple of 2", (double)v);
                r->N[seen_n++] = v;
                break;
            }
            case 's':
                r->t0 = atof(optarg);
                if (r->t0 < 0) die_num("The integration start time [%lf] must be a positive", r->t0);
                break;
            case 'e':
                r->T = atof(optarg);
                if (r->T < 0) die_num("The integration end time [%lf] must be a positive", r->T);
                if (r->T < r->t0) die_num("The provided end time [%lf] must be greater than the initial time", r->T);
                break;
            case 'h':
                if (seen_h++ == 0) {
                    r->dt = atof(optarg);
                    if (r->dt <= 0) die_num("The provided timestep: [%lf] must be strictly positive", r->dt);
                } else {
                    r->adapt_step = flag01(optarg, "Adaptive stepping");
                }
                break;
            case 'c':
                if (seen_c++ == 0) {
                    r->cfl_cond = flag01(optarg, "CFL condition");
                } else {
                    r->cfl_const = atof(optarg);
                    if (r->cfl_const <= 0) die_num("The provided CFL Constant: [%lf] must be strictly positive", r->cfl_const);
                }
                break;
            case 'v':
                if (seen_v == 0) {
                    r->nu = atof(optarg);
                    if (r->nu < 0) die_num("The provided viscosity: [%lf] must be positive", r->nu);
                } else if (seen_v == 1) {
                    r->hyper_flag = flag01(optarg, "Hyperviscosity");
                } else {
                    r->hyper_pow = atof(optarg);
                    if (r->hyper_pow <= 0.0) die_num("The provided hyperviscosity power: [%lf] must be strictly positive", r->hyper_pow);
                }
                seen_v++;
                break;
            case 'd':
                if (seen_d == 0) {
                    r->ekmn_alpha = atof(optarg);
                    if (r->ekmn_alpha < 0) die_num("The provided Ekman Drag: [%lf] must be positive", r->ekmn_alpha);
                } else if (seen_d == 1) {
                    r->ekmn_flag = flag01(optarg, "Ekman Drag");
                } else {
                    r->ekmn_pow = atof(optarg);
                    if (r->ekmn_pow > 0.0) die_num("The provided Hypodiffusivity power: [%lf] must be negative or zero", r->ekmn_pow);
                }
                seen_d++;
                break;
            case 'i':
                copy(r->u0, sizeof(r->u0), in_list(optarg, k_initial) ? optarg : "NONE");
                break;
            case 't':
                copy(r->output_tag, sizeof(r->output_tag), optarg);
                break;
            case 'T':
                if (seen_T++ == 0) {
                    r->trans_iters = flag01(optarg, "transient iterations");
                } else {
                    r->trans_frac = atof(optarg);
                    if (r->trans_frac >= 1.0 || r->trans_frac <= 0.0)
                        die_num("Incorrect transient iterations fraction: [%lf] Must be between 0 and 1", r->trans_frac);
                }
                break;
            case 'p':
                r->save_every = atoi(optarg);
                if (r->save_every <= 0) die_num("The save interval [%g] must be a positive number of iterations", (double)r->save_every);
                break;
            case 'f':
                if (seen_f == 0) {
                    if (in_list(optarg, k_forcing)) {
                        copy(r->forcing, sizeof(r->forcing), optarg);
                        seen_f = 1;
                    }
                } else if (seen_f == 1) {
                    r->force_k = atoi(optarg);
                    seen_f = 2;
                } else {
                    r->force_scale = atof(optarg);
                }
                break;
            case 'z':
                copy(r->input_file, sizeof(r->input_file), optarg);
                if (access(r->input_file, F_OK) != 0)
                    die_str("The input file [%s] cannot be found, please ensure correct path to file is specified.", r->input_file);
                break;
            case OPT_INTEGRATOR:
                if (!strcmp(optarg, "RK4CN")) r->integrator = NS2D_RK4CN;
                else if (!strcmp(optarg, "RK4")) r->integrator = NS2D_RK4;
                else if (!strcmp(optarg, "AB4")) r->integrator = NS2D_AB4;
                else if (!strcmp(optarg, "DP5")) r->integrator = NS2D_DP5;
                else die_str("Unknown integrator [%s]", optarg);
                break;
            case OPT_DEALIAS:
                if (!strcmp(optarg, "23")) r->dealias = NS2D_DEALIAS_23;
                else if (!strcmp(optarg, "HOU_LI")) r->dealias = NS2D_DEALIAS_HOU_LI;
                else die_str("Unknown dealiasing [%s]", optarg);
                break;
            case OPT_PRECISION:
                if (!strcmp(optarg, "FP64")) r->precision = NS2D_FP64;
                else if (!strcmp(optarg, "FP32")) r->precision = NS2D_FP32;
                else die_str("Unknown precision [%s]", optarg);
                break;
            case OPT_DEVICE:
                r->device = atoi(optarg);
                break;
            case OPT_NO_QUIRKS:
                r->quirks = 0;
                break;
            case OPT_DRY_RUN:
                r->dry_run = 1;
                break;
            case OPT_QUIET:
                r->quiet = 1;
                break;
            case OPT_PHASE_ONLY:
                r->phase_only = 1;
                break;
            default:
                usage_and_exit();
        }
    }
    /* the phase-only reset exists in RK4Step only (solver.c:822-857) */
    if (r->phase_only && r->integrator != NS2D_RK4CN && r->integrator != NS2D_RK4)
        die_str("--phase-only needs --integrator=RK4CN or RK4%s", "");
}
