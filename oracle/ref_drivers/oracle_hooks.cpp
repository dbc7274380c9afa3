/*
 * Test infrastructure (oracle side only): definitions for the hooks declared
 * in fullprec_hook.h. Linked into the reference apps built under oracle/_ref.
 *
 * - oracle_printf / oracle_fprintf: printf-compatible; every floating
 *   conversion (%e %E %f %g with any flags/width/precision/length) is printed
 *   as "%.17E" so that the doubles the reference app reports survive the
 *   round trip through text exactly.
 * - oracle_exit: if ORACLE_DUMP_DIR is set, writes each dat of the OPS
 *   instance (reference host layout: x fastest, halos and x-padding included)
 *   to <dir>/<name>.bin and its metadata to <dir>/<name>.meta, then calls the
 *   reference ops_exit (ops/c/src/core/ops_dummy_singlenode.cpp).
 */
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "ops_lib_core.h"
#include "ops_internal2.h"
#include "ops_instance.h"

static void widen_vfprintf(FILE *out, const char *fmt, va_list ap) {
  const char *p = fmt;
  while (*p) {
    if (*p != '%') { fputc(*p++, out); continue; }
    const char *start = p++;
    if (*p == '%') { fputc('%', out); p++; continue; }
    while (*p && strchr("-+ #0", *p)) p++;
    while (*p >= '0' && *p <= '9') p++;
    if (*p == '*') { p++; }
    if (*p == '.') { p++; while (*p >= '0' && *p <= '9') p++; }
    int lng = 0;
    while (*p && strchr("hlLqjzt", *p)) { if (*p == 'l') lng++; p++; }
    char conv = *p ? *p++ : 0;
    std::string spec(start, p - start);
    switch (conv) {
      case 'e': case 'E': case 'f': case 'F': case 'g': case 'G':
        fprintf(out, "%.17E", va_arg(ap, double));
        break;
      case 'd': case 'i':
        if (lng >= 2) fprintf(out, spec.c_str(), va_arg(ap, long long));
        else if (lng == 1) fprintf(out, spec.c_str(), va_arg(ap, long));
        else fprintf(out, spec.c_str(), va_arg(ap, int));
        break;
      case 'u': case 'x': case 'X': case 'o':
        if (lng >= 2) fprintf(out, spec.c_str(), va_arg(ap, unsigned long long));
        else if (lng == 1) fprintf(out, spec.c_str(), va_arg(ap, unsigned long));
        else fprintf(out, spec.c_str(), va_arg(ap, unsigned));
        break;
      case 's': fprintf(out, spec.c_str(), va_arg(ap, const char *)); break;
      case 'c': fprintf(out, spec.c_str(), va_arg(ap, int)); break;
      case 'p': fprintf(out, spec.c_str(), va_arg(ap, void *)); break;
      default: fputs(spec.c_str(), out); break;
    }
  }
}

void oracle_printf(const char *format, ...) {
  va_list ap;
  va_start(ap, format);
  widen_vfprintf(stdout, format, ap);
  va_end(ap);
  fflush(stdout);
}

void oracle_fprintf(FILE *stream, const char *format, ...) {
  va_list ap;
  va_start(ap, format);
  widen_vfprintf(stream, format, ap);
  va_end(ap);
}

void oracle_exit() {
  const char *dir = getenv("ORACLE_DUMP_DIR");
  if (dir != NULL) {
    OPS_instance *inst = OPS_instance::getOPSInstance();
    ops_dat_entry *item;
    TAILQ_FOREACH(item, &(inst->OPS_dat_list), entries) {
      ops_dat dat = item->dat;
      ops_get_data(dat);
      std::string base = std::string(dir) + "/" + dat->name;
      FILE *fb = fopen((base + ".bin").c_str(), "wb");
      if (fb) { fwrite(dat->data, 1, dat->mem, fb); fclose(fb); }
      FILE *fm = fopen((base + ".meta").c_str(), "w");
      if (fm) {
        int nd = dat->block->dims;
        fprintf(fm, "dims %d elem_size %d type %s\n", nd, dat->elem_size, dat->type);
        fprintf(fm, "size"); for (int d = 0; d < nd; d++) fprintf(fm, " %d", dat->size[d]); fprintf(fm, "\n");
        fprintf(fm, "d_m"); for (int d = 0; d < nd; d++) fprintf(fm, " %d", dat->d_m[d]); fprintf(fm, "\n");
        fprintf(fm, "d_p"); for (int d = 0; d < nd; d++) fprintf(fm, " %d", dat->d_p[d]); fprintf(fm, "\n");
        fprintf(fm, "x_pad %d\n", dat->x_pad);
        fclose(fm);
      }
    }
  }
  ops_exit();
}
