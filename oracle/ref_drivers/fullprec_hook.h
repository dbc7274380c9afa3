/*
 * Test infrastructure (oracle side only): forced-include header for the
 * reference OPS apps built into oracle/_ref.
 *
 * The reference apps print their field summaries and timestep lines with
 * 3-4 significant digits (apps/c/CloverLeaf/field_summary.cpp:75-77,
 * apps/c/CloverLeaf/time_step.cpp:116-121). Parity checks need the full
 * double, so every ops_printf / ops_fprintf issued by the APP code is routed
 * through a formatter that widens each floating conversion to "%.17E".
 * The reference library itself is compiled without this header, so its own
 * diagnostics are untouched. ops_exit is routed through a hook that, when
 * ORACLE_DUMP_DIR is set, writes every declared dat (halo included, in the
 * reference's own host layout) to <dir>/<name>.bin before the real ops_exit.
 *
 * Nothing of the reference source is modified or copied; this header only
 * renames three call targets at compile time.
 */
#ifndef ORACLE_FULLPREC_HOOK_H
#define ORACLE_FULLPREC_HOOK_H
#include <stdio.h>
void oracle_printf(const char *format, ...);
void oracle_fprintf(FILE *stream, const char *format, ...);
void oracle_exit();
#define ops_printf oracle_printf
#define ops_fprintf oracle_fprintf
#define ops_exit oracle_exit
#endif
