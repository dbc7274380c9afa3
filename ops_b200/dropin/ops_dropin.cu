// The reference OPS C++ API (the mangled ops_* symbols an OPS application
// and its translated code link against) implemented on the OPS-B200
// runtime. Compiled against the reference's own public headers, so every
// struct an application reads (ops_block_core, ops_dat_core,
// ops_stencil_core, ops_arg, ops_reduction_core: ops/c/include/
// ops_lib_core.h:183-552) has the reference's layout; the runtime's own
// objects are found through each struct's `index`.
//
// Semantics follow the reference's single-process backends (ops/c/src/core/
// ops_lib_core.cpp, ops_lazy.cpp, ops_dummy_singlenode.cpp,
// ops_device_singlenode_common.cpp), cited per function. There is one
// device path and no host fallback: ops_init fails without a GPU.
#include <sys/time.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "ops_lib_core.h"
#include "ops_instance.h"
#include "ops_util.h"
#include "ops_checkpointing.h"
#include "ops_dropin.h"

namespace {
using opsb::Runtime;

// Every struct handed out, freed by ops_exit.
struct Handles {
  std::vector<ops_block_core *> blocks;
  std::vector<ops_dat_core *> dats;
  std::vector<ops_stencil_core *> stencils;
  std::vector<ops_reduction_core *> reductions;
  std::vector<ops_halo_core *> halos;
  std::vector<ops_halo_group_core *> groups;
};
Handles &handles() {
  static Handles h;
  return h;
}

char *dup(const char *s) {
  const char *t = s ? s : "";
  char *r = static_cast<char *>(malloc(strlen(t) + 1));
  strcpy(r, t);
  return r;
}

// A runtime error as the reference reports it: an OPSException
// (ops/c/include/ops_exceptions.h:46-77), OPS_RUNTIME_ERROR for device
// failures.
[[noreturn]] void rethrow(const opsb::Error &e) {
  OPSException ex(e.code == opsb::E_ARG ? OPS_INVALID_ARGUMENT : OPS_RUNTIME_ERROR);
  ex << e.msg;
  throw ex;
}
template <class F>
auto guarded(F &&f) -> decltype(f()) {
  try {
    return f();
  } catch (const opsb::Error &e) {
    rethrow(e);
  }
}

Runtime &rt() {
  if (!Runtime::exists()) {
    OPSException ex(OPS_RUNTIME_ERROR);
    ex << "ops_init has not been called";
    throw ex;
  }
  return Runtime::get();
}

// ops_printf / ops_fprintf: OPS_B200_PRINT_FULL=1 prints every floating
// conversion with 17 significant digits ("%.17E"), so that the values an
// application reports can be compared exactly.
bool full_precision() {
  static const bool f = getenv("OPS_B200_PRINT_FULL") && atoi(getenv("OPS_B200_PRINT_FULL")) != 0;
  return f;
}
void print_formatted(FILE *out, const char *fmt, va_list ap) {
  if (!full_precision()) {
    vfprintf(out, fmt, ap);
    return;
  }
  for (const char *p = fmt; *p;) {
    if (*p != '%') {
      fputc(*p++, out);
      continue;
    }
    const char *start = p++;
    if (*p == '%') {
      fputc('%', out);
      p++;
      continue;
    }
    while (*p && strchr("-+ #0", *p)) p++;
    while (*p >= '0' && *p <= '9') p++;
    if (*p == '.') {
      p++;
      while (*p >= '0' && *p <= '9') p++;
    }
    int longs = 0;
    while (*p && strchr("hlLqjzt", *p)) longs += (*p++ == 'l');
    const char conv = *p ? *p++ : 0;
    const std::string spec(start, p - start);
    switch (conv) {
      case 'e': case 'E': case 'f': case 'F': case 'g': case 'G':
        fprintf(out, "%.17E", va_arg(ap, double));
        break;
      case 'd': case 'i':
        if (longs >= 2) fprintf(out, spec.c_str(), va_arg(ap, long long));
        else if (longs == 1) fprintf(out, spec.c_str(), va_arg(ap, long));
        else fprintf(out, spec.c_str(), va_arg(ap, int));
        break;
      case 'u': case 'x': case 'X': case 'o':
        if (longs >= 2) fprintf(out, spec.c_str(), va_arg(ap, unsigned long long));
        else if (longs == 1) fprintf(out, spec.c_str(), va_arg(ap, unsigned long));
        else fprintf(out, spec.c_str(), va_arg(ap, unsigned));
        break;
      case 's': fprintf(out, spec.c_str(), va_arg(ap, const char *)); break;
      case 'c': fprintf(out, spec.c_str(), va_arg(ap, int)); break;
      case 'p': fprintf(out, spec.c_str(), va_arg(ap, void *)); break;
      default: fputs(spec.c_str(), out); break;
    }
  }
}

// The host copy of a dat in the reference's host layout (x fastest, halos
// included, no padding: ops_dat_core::x_pad = 0).
size_t host_bytes(const ops_dat_core *d) {
  size_t n = (size_t)d->elem_size;
  for (int i = 0; i < d->block->dims; i++) n *= (size_t)d->size[i];
  return n;
}
void refresh_host(ops_dat_core *d) { guarded([&] { rt().dat_fetch_data(d->index, d->data, host_bytes(d)); }); }

// OPS_B200_DUMP_DIR: at ops_exit every dat is written to <dir>/<name>.bin in
// the host layout above (for comparing a run with another build).
void dump_dats() {
  const char *dir = getenv("OPS_B200_DUMP_DIR");
  if (!dir) return;
  for (ops_dat_core *d : handles().dats) {
    refresh_host(d);
    std::string name(d->name);
    while (!name.empty() && name.back() == ' ') name.pop_back();
    while (!name.empty() && name.front() == ' ') name.erase(0, 1);
    const std::string path = std::string(dir) + "/" + name + ".bin";
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) continue;
    fwrite(d->data, 1, host_bytes(d), f);
    fclose(f);
  }
}
}  // namespace

// ---------------------------------------------------------------------------
// Instance and lifecycle (ops/c/src/core/ops_dummy_singlenode.cpp:979,
// ops_instance.cpp:37). The runtime is the process's single instance. The
// OPS_instance the reference's inline templates pass along and that
// applications read settings from (OPS_diags, clover_leaf.cpp's power
// counters) is zeroed storage of the reference's layout whose plain fields
// ops_init sets; nothing in it is constructed or owned.
// ---------------------------------------------------------------------------
namespace {
alignas(OPS_instance) unsigned char g_instance_storage[sizeof(OPS_instance)];
}
OPS_instance *OPS_instance::getOPSInstance() { return reinterpret_cast<OPS_instance *>(g_instance_storage); }

// Row and plane sizes the legacy kernel style addresses through
// (OPS_ACC<n>(x, y) = x + xdim<n> * y, ops/c/include/ops_macros.h:2785-2870).
// The device functors the sm100a target makes from such kernels use
// accessors instead; these definitions only satisfy the host copies of the
// kernel functions that an application's translated files still compile.
extern "C" {
int xdim0, xdim1, xdim2, xdim3, xdim4, xdim5, xdim6, xdim7, xdim8, xdim9, xdim10, xdim11, xdim12, xdim13, xdim14,
    xdim15, xdim16, xdim17, xdim18, xdim19, xdim20, xdim21, xdim22, xdim23, xdim24, xdim25, xdim26, xdim27, xdim28,
    xdim29, xdim30, xdim31, xdim32, xdim33, xdim34, xdim35, xdim36, xdim37, xdim38, xdim39, xdim40, xdim41, xdim42,
    xdim43, xdim44, xdim45, xdim46, xdim47, xdim48, xdim49, xdim50, xdim51, xdim52, xdim53, xdim54, xdim55, xdim56,
    xdim57, xdim58, xdim59, xdim60, xdim61, xdim62, xdim63, xdim64, xdim65, xdim66, xdim67, xdim68, xdim69, xdim70,
    xdim71, xdim72, xdim73, xdim74, xdim75, xdim76, xdim77, xdim78, xdim79, xdim80, xdim81, xdim82, xdim83, xdim84,
    xdim85, xdim86, xdim87, xdim88, xdim89, xdim90, xdim91, xdim92, xdim93, xdim94, xdim95, xdim96, xdim97, xdim98,
    xdim99;
int ydim0, ydim1, ydim2, ydim3, ydim4, ydim5, ydim6, ydim7, ydim8, ydim9, ydim10, ydim11, ydim12, ydim13, ydim14,
    ydim15, ydim16, ydim17, ydim18, ydim19, ydim20, ydim21, ydim22, ydim23, ydim24, ydim25, ydim26, ydim27, ydim28,
    ydim29, ydim30, ydim31, ydim32, ydim33, ydim34, ydim35, ydim36, ydim37, ydim38, ydim39, ydim40, ydim41, ydim42,
    ydim43, ydim44, ydim45, ydim46, ydim47, ydim48, ydim49, ydim50, ydim51, ydim52, ydim53, ydim54, ydim55, ydim56,
    ydim57, ydim58, ydim59, ydim60, ydim61, ydim62, ydim63, ydim64, ydim65, ydim66, ydim67, ydim68, ydim69, ydim70,
    ydim71, ydim72, ydim73, ydim74, ydim75, ydim76, ydim77, ydim78, ydim79, ydim80, ydim81, ydim82, ydim83, ydim84,
    ydim85, ydim86, ydim87, ydim88, ydim89, ydim90, ydim91, ydim92, ydim93, ydim94, ydim95, ydim96, ydim97, ydim98,
    ydim99;
int zdim0, zdim1, zdim2, zdim3, zdim4, zdim5, zdim6, zdim7, zdim8, zdim9, zdim10, zdim11, zdim12, zdim13, zdim14,
    zdim15, zdim16, zdim17, zdim18, zdim19, zdim20, zdim21, zdim22, zdim23, zdim24, zdim25, zdim26, zdim27, zdim28,
    zdim29, zdim30, zdim31, zdim32, zdim33, zdim34, zdim35, zdim36, zdim37, zdim38, zdim39, zdim40, zdim41, zdim42,
    zdim43, zdim44, zdim45, zdim46, zdim47, zdim48, zdim49, zdim50, zdim51, zdim52, zdim53, zdim54, zdim55, zdim56,
    zdim57, zdim58, zdim59, zdim60, zdim61, zdim62, zdim63, zdim64, zdim65, zdim66, zdim67, zdim68, zdim69, zdim70,
    zdim71, zdim72, zdim73, zdim74, zdim75, zdim76, zdim77, zdim78, zdim79, zdim80, zdim81, zdim82, zdim83, zdim84,
    zdim85, zdim86, zdim87, zdim88, zdim89, zdim90, zdim91, zdim92, zdim93, zdim94, zdim95, zdim96, zdim97, zdim98,
    zdim99;
int udim0, udim1, udim2, udim3, udim4, udim5, udim6, udim7, udim8, udim9, udim10, udim11, udim12, udim13, udim14,
    udim15, udim16, udim17, udim18, udim19, udim20, udim21, udim22, udim23, udim24, udim25, udim26, udim27, udim28,
    udim29, udim30, udim31, udim32, udim33, udim34, udim35, udim36, udim37, udim38, udim39, udim40, udim41, udim42,
    udim43, udim44, udim45, udim46, udim47, udim48, udim49, udim50, udim51, udim52, udim53, udim54, udim55, udim56,
    udim57, udim58, udim59, udim60, udim61, udim62, udim63, udim64, udim65, udim66, udim67, udim68, udim69, udim70,
    udim71, udim72, udim73, udim74, udim75, udim76, udim77, udim78, udim79, udim80, udim81, udim82, udim83, udim84,
    udim85, udim86, udim87, udim88, udim89, udim90, udim91, udim92, udim93, udim94, udim95, udim96, udim97, udim98,
    udim99;
}

// GPU power sampling is not part of this backend (NVML is out of scope).
void OPS_instance::reset_power_counters() {}

// The reference's allocation helpers (ops/c/include/ops_util.h), used by
// application code.
void *xmalloc(size_t size) {
  void *p = size ? malloc(size) : nullptr;
  if (size && !p) {
    OPSException ex(OPS_RUNTIME_ERROR);
    ex << "xmalloc: out of host memory";
    throw ex;
  }
  return p;
}
void *xrealloc(void *ptr, size_t size) {
  void *p = realloc(ptr, size);
  if (size && !p) {
    OPSException ex(OPS_RUNTIME_ERROR);
    ex << "xrealloc: out of host memory";
    throw ex;
  }
  return p;
}
void *xcalloc(size_t number, size_t size) {
  void *p = calloc(number, size);
  if (number && size && !p) {
    OPSException ex(OPS_RUNTIME_ERROR);
    ex << "xcalloc: out of host memory";
    throw ex;
  }
  return p;
}

void ops_init(const int argc, const char *const argv[], const int diags_level) {
  (void)argc;
  (void)argv;
  int device = 0;
  if (const char *d = getenv("OPS_B200_DEVICE")) device = atoi(d);
  guarded([&] { Runtime::get().init(device, diags_level); });
  OPS_instance::getOPSInstance()->OPS_diags = diags_level;
}

void ops_exit() {
  if (!Runtime::exists()) return;
  dump_dats();
  guarded([&] { Runtime::get().execute(); });
  Handles &h = handles();
  for (ops_dat_core *d : h.dats) {
    free(d->data);
    free(const_cast<char *>(d->name));
    free(const_cast<char *>(d->type));
    delete d;
  }
  for (ops_block_core *b : h.blocks) {
    free(const_cast<char *>(b->name));
    delete b;
  }
  for (ops_stencil_core *s : h.stencils) {
    free(s->stencil);
    free(s->stride);
    free(s->mgrid_stride);
    free(const_cast<char *>(s->name));
    delete s;
  }
  for (ops_reduction_core *r : h.reductions) {
    free(r->data);
    free(r->type);
    free(r->name);
    delete r;
  }
  for (ops_halo_core *x : h.halos) delete x;
  for (ops_halo_group_core *g : h.groups) {
    free(g->halos);
    delete g;
  }
  h = Handles();
  Runtime::destroy();
}

// ops_init_backend is emitted by the translator's backend targets; the
// sm100a target emits it too (it has nothing to set up).
void ops_set_soa(const int soa_val) {
  if (soa_val != 0) {
    OPSException ex(OPS_NOT_IMPLEMENTED);
    ex << "OPS-B200 supports one-component dats only (no structure-of-arrays dats)";
    throw ex;
  }
}

// ---------------------------------------------------------------------------
// Declarations (ops/c/src/core/ops_lib_core.cpp:445-548, 640-832, 1119).
// ---------------------------------------------------------------------------
ops_block ops_decl_block(int dims, const char *name) {
  return guarded([&] {
    ops_block_core *b = new ops_block_core();
    b->index = rt().decl_block(dims, name);
    b->dims = dims;
    b->name = dup(name);
    b->instance = OPS_instance::getOPSInstance();
    handles().blocks.push_back(b);
    return b;
  });
}

ops_dat ops_decl_dat_char(ops_block block, int dim, int *size, int *base, int *d_m, int *d_p, int *stride, char *data,
                          int type_size, char const *type, char const *name) {
  (void)stride;  // the coarsening factor of multigrid dats steers the reference's MPI decomposition only
  return guarded([&] {
    if (!block) throw opsb::Error(opsb::E_ARG, "ops_decl_dat: NULL block");
    ops_dat_core *d = new ops_dat_core();
    d->index = rt().decl_dat(block->index, dim, size, base, d_m, d_p, data, type_size, type, name);
    const opsb::Dat &r = rt().dat(d->index);
    d->block = block;
    d->dim = dim;
    d->type_size = type_size;
    d->elem_size = dim * type_size;
    for (int i = 0; i < OPS_MAX_DIM; i++) {
      const bool in = i < block->dims;
      d->size[i] = in ? r.size[i] : 1;
      d->base[i] = in ? base[i] : 0;
      d->d_m[i] = in ? d_m[i] : 0;
      d->d_p[i] = in ? d_p[i] : 0;
      d->stride[i] = 1;
    }
    d->x_pad = 0;
    d->mem = host_bytes(d);
    d->data = static_cast<char *>(calloc(d->mem, 1));
    if (data) memcpy(d->data, data, d->mem);
    d->data_d = r.data_d;
    d->name = dup(name);
    d->type = dup(type);
    d->user_managed = data != nullptr;
    d->dirty_hd = 0;
    handles().dats.push_back(d);
    return d;
  });
}

ops_dat_core::~ops_dat_core() {}

void ops_free_dat(ops_dat dat) {
  (void)dat;  // the storage is released with the instance (ops_exit)
}

static ops_stencil make_stencil(int h, int dims, int points, const int *sten, const int *stride, const int *mgrid,
                                int type, char const *name) {
  ops_stencil_core *s = new ops_stencil_core();
  s->index = h;
  s->dims = dims;
  s->points = points;
  s->name = dup(name);
  s->stencil = static_cast<int *>(malloc(sizeof(int) * dims * points));
  memcpy(s->stencil, sten, sizeof(int) * dims * points);
  s->stride = static_cast<int *>(malloc(sizeof(int) * dims));
  s->mgrid_stride = static_cast<int *>(malloc(sizeof(int) * dims));
  for (int i = 0; i < dims; i++) {
    s->stride[i] = stride ? stride[i] : 1;
    s->mgrid_stride[i] = mgrid ? mgrid[i] : 1;
  }
  s->type = type;
  handles().stencils.push_back(s);
  return s;
}

ops_stencil ops_decl_stencil(int dims, int points, int *sten, char const *name) {
  return guarded([&] {
    const int h = rt().decl_stencil(dims, points, sten, nullptr, name);
    return make_stencil(h, dims, points, sten, nullptr, nullptr, 0, name);
  });
}

ops_stencil ops_decl_strided_stencil(int dims, int points, int *sten, int *stride, char const *name) {
  return guarded([&] {
    const int h = rt().decl_stencil(dims, points, sten, stride, name);
    return make_stencil(h, dims, points, sten, stride, nullptr, 0, name);
  });
}

ops_stencil ops_decl_restrict_stencil(int dims, int points, int *sten, int *stride, char const *name) {
  return guarded([&] {
    const int h = rt().decl_mgrid_stencil(dims, points, sten, stride, 2, name);
    return make_stencil(h, dims, points, sten, nullptr, stride, 2, name);
  });
}

ops_stencil ops_decl_prolong_stencil(int dims, int points, int *sten, int *stride, char const *name) {
  return guarded([&] {
    const int h = rt().decl_mgrid_stencil(dims, points, sten, stride, 1, name);
    return make_stencil(h, dims, points, sten, nullptr, stride, 1, name);
  });
}

// ---------------------------------------------------------------------------
// Arguments (ops/c/src/core/ops_lib_core.cpp:856, 1047-1118). A reduction is
// a global argument whose data is the handle (ops_arg_reduce_core).
// ---------------------------------------------------------------------------
ops_arg ops_arg_dat(ops_dat dat, int dim, ops_stencil stencil, char const *type, ops_access acc) {
  return ops_arg_dat_opt(dat, dim, stencil, type, acc, 1);
}

ops_arg ops_arg_dat_opt(ops_dat dat, int dim, ops_stencil stencil, char const *type, ops_access acc, int flag) {
  (void)type;
  ops_arg a;
  memset(&a, 0, sizeof(a));
  a.dat = dat;
  a.stencil = stencil;
  a.dim = dim;
  a.elem_size = dat ? dat->type_size : 0;
  a.data = dat ? dat->data : nullptr;
  a.data_d = dat ? dat->data_d : nullptr;
  a.acc = acc;
  a.argtype = OPS_ARG_DAT;
  a.opt = flag ? 1 : 0;
  return a;
}

ops_arg ops_arg_idx() {
  ops_arg a;
  memset(&a, 0, sizeof(a));
  a.argtype = OPS_ARG_IDX;
  a.opt = 1;
  return a;
}

ops_arg ops_arg_gbl_char(char *data, int dim, int size, ops_access acc) {
  ops_arg a;
  memset(&a, 0, sizeof(a));
  a.data = data;
  a.dim = dim;
  a.elem_size = size;
  a.acc = acc;
  a.argtype = OPS_ARG_GBL;
  a.opt = 1;
  return a;
}

ops_arg ops_arg_reduce(ops_reduction handle, int dim, const char *type, ops_access acc) {
  (void)type;
  ops_arg a;
  memset(&a, 0, sizeof(a));
  a.data = reinterpret_cast<char *>(handle);
  a.dim = dim;
  a.elem_size = handle ? handle->size / (dim > 0 ? dim : 1) : 0;
  a.acc = acc;
  a.argtype = OPS_ARG_GBL;
  a.opt = 1;
  return a;
}

ops_reduction ops_decl_reduction_handle(int size, const char *type, const char *name) {
  return guarded([&] {
    ops_reduction_core *r = new ops_reduction_core();
    r->index = rt().decl_reduction(size, type, name);
    r->size = size;
    r->data = static_cast<char *>(calloc((size_t)size, 1));
    r->initialized = 0;
    r->acc = OPS_READ;
    r->type = dup(type);
    r->name = dup(name);
    r->instance = OPS_instance::getOPSInstance();
    handles().reductions.push_back(r);
    return r;
  });
}

// ops_reduction_result_char (ops/c/src/core/ops_lib_core.cpp:1143): runs the
// queued loops, copies the value out and resets the handle.
void ops_reduction_result_char(ops_reduction_core *handle, int type_size, char *ptr) {
  (void)type_size;
  guarded([&] {
    rt().reduction_result(handle->index, handle->data);
    memcpy(ptr, handle->data, (size_t)handle->size);
    handle->initialized = 0;
  });
}

// ---------------------------------------------------------------------------
// Loops and constants (called by the code the sm100a target generates).
// ---------------------------------------------------------------------------
const opsb::LoopInfo *opsb_dropin_find_loop(const char *kernel) {
  const opsb::LoopInfo *li = Runtime::find_loop(kernel);
  if (!li) {
    OPSException ex(OPS_RUNTIME_ERROR);
    ex << "no sm100a loop kernel registered as " << kernel;
    throw ex;
  }
  return li;
}

void opsb_dropin_par_loop(const opsb::LoopInfo *loop, char const *name, ops_block block, int dim, int *range,
                          ops_arg *args, int nargs) {
  guarded([&] {
    opsb::Arg conv[OPSB_MAX_ARGS];
    if (nargs > OPSB_MAX_ARGS) throw opsb::Error(opsb::E_ARG, "ops_par_loop: too many arguments");
    for (int i = 0; i < nargs; i++) {
      const ops_arg &a = args[i];
      switch (a.argtype) {
        case OPS_ARG_DAT:
          if (!a.dat || !a.stencil) throw opsb::Error(opsb::E_ARG, std::string("ops_par_loop ") + name + ": NULL dat");
          conv[i] = opsb::arg_dat_opt(a.dat->index, a.dim, a.stencil->index, a.acc, a.opt);
          break;
        case OPS_ARG_GBL:
          if (a.acc == OPS_READ) {
            conv[i] = opsb::arg_gbl(a.data, a.dim, a.elem_size, opsb::ACC_READ);
          } else {
            ops_reduction h = reinterpret_cast<ops_reduction>(a.data);
            conv[i] = opsb::arg_reduce(h->index, a.dim, a.acc);
            h->initialized = 1;
            h->acc = a.acc;
          }
          break;
        case OPS_ARG_IDX:
          conv[i] = opsb::arg_idx();
          break;
        default:
          throw opsb::Error(opsb::E_ARG, "ops_par_loop: unknown argument type");
      }
    }
    rt().par_loop(loop, name, block->index, dim, range, conv, nargs);
  });
}

cudaStream_t opsb_dropin_const_begin() {
  return guarded([&] {
    rt().execute();
    return rt().stream();
  });
}

void opsb_dropin_const_done(cudaError_t copy_status, const char *name) {
  cudaError_t e = copy_status;
  if (e == cudaSuccess) e = cudaStreamSynchronize(rt().stream());
  if (e != cudaSuccess) {
    OPSException ex(OPS_RUNTIME_ERROR);
    ex << "ops_decl_const " << name << ": " << cudaGetErrorString(e);
    throw ex;
  }
}

void ops_execute(OPS_instance *instance) {
  (void)instance;
  guarded([&] { rt().execute(); });
}

// ---------------------------------------------------------------------------
// Halos between blocks (ops/c/src/core/ops_lib_core.cpp:998-1040,
// ops_device_singlenode_common.cpp:262-346).
// ---------------------------------------------------------------------------
ops_halo ops_decl_halo(ops_dat from, ops_dat to, int *iter_size, int *from_base, int *to_base, int *from_dir,
                       int *to_dir) {
  return guarded([&] {
    ops_halo_core *h = new ops_halo_core();
    h->index = rt().decl_halo(from->index, to->index, iter_size, from_base, to_base, from_dir, to_dir);
    h->from = from;
    h->to = to;
    const int nd = from->block->dims;
    for (int i = 0; i < OPS_MAX_DIM; i++) {
      h->iter_size[i] = i < nd ? iter_size[i] : 1;
      h->from_base[i] = i < nd ? from_base[i] : 0;
      h->to_base[i] = i < nd ? to_base[i] : 0;
      h->from_dir[i] = i < nd ? from_dir[i] : i + 1;
      h->to_dir[i] = i < nd ? to_dir[i] : i + 1;
    }
    handles().halos.push_back(h);
    return h;
  });
}

ops_halo_group ops_decl_halo_group(int nhalos, ops_halo *halos) {
  return guarded([&] {
    std::vector<int> idx(nhalos);
    for (int i = 0; i < nhalos; i++) idx[i] = halos[i]->index;
    ops_halo_group_core *g = new ops_halo_group_core();
    g->index = rt().decl_halo_group(nhalos, idx.data());
    g->nhalos = nhalos;
    g->halos = static_cast<ops_halo *>(malloc(sizeof(ops_halo) * (nhalos > 0 ? nhalos : 1)));
    for (int i = 0; i < nhalos; i++) g->halos[i] = halos[i];
    g->instance = OPS_instance::getOPSInstance();
    handles().groups.push_back(g);
    return g;
  });
}

void ops_halo_transfer(ops_halo_group group) {
  guarded([&] { rt().halo_transfer(group->index); });
}

// ---------------------------------------------------------------------------
// Data access (ops/c/src/core/ops_dummy_singlenode.cpp:611-850,
// ops_device_singlenode_common.cpp:109-260). part is always 0 (one process).
// ---------------------------------------------------------------------------
void ops_get_data(ops_dat dat) { refresh_host(dat); }

void ops_dat_fetch_data(ops_dat dat, int part, char *data) {
  (void)part;
  guarded([&] { rt().dat_fetch_data(dat->index, data, host_bytes(dat)); });
}

void ops_dat_fetch_data_memspace(ops_dat dat, int part, char *data, ops_memspace memspace) {
  if (memspace != OPS_HOST) {
    OPSException ex(OPS_NOT_IMPLEMENTED);
    ex << "ops_dat_fetch_data_memspace: only OPS_HOST destinations";
    throw ex;
  }
  ops_dat_fetch_data(dat, part, data);
}

void ops_dat_set_data(ops_dat dat, int part, char *data) {
  (void)part;
  guarded([&] { rt().dat_set_data(dat->index, data, host_bytes(dat)); });
}

void ops_dat_set_data_memspace(ops_dat dat, int part, char *data, ops_memspace memspace) {
  if (memspace != OPS_HOST) {
    OPSException ex(OPS_NOT_IMPLEMENTED);
    ex << "ops_dat_set_data_memspace: only OPS_HOST sources";
    throw ex;
  }
  ops_dat_set_data(dat, part, data);
}

int ops_dat_get_local_npartitions(ops_dat dat) {
  (void)dat;
  return 1;
}
int ops_dat_get_global_npartitions(ops_dat dat) {
  (void)dat;
  return 1;
}

void ops_dat_get_extents(ops_dat dat, int part, int *disp, int *size) {
  (void)part;
  for (int i = 0; i < dat->block->dims; i++) {
    if (disp) disp[i] = 0;
    if (size) size[i] = dat->size[i];
  }
}

// The raw pointer addresses the dat's first point (logical base + d_m); the
// row stride the runtime reports includes its 128-byte row padding.
void ops_dat_get_raw_metadata(ops_dat dat, int part, int *disp, int *size, int *stride, int *d_m, int *d_p) {
  (void)part;
  const opsb::Dat &r = guarded([&]() -> const opsb::Dat & { return rt().dat(dat->index); });
  const int nd = dat->block->dims;
  for (int i = 0; i < nd; i++) {
    if (disp) disp[i] = 0;
    if (size) size[i] = dat->size[i];
    if (d_m) d_m[i] = dat->d_m[i];
    if (d_p) d_p[i] = dat->d_p[i];
  }
  if (stride) {
    stride[0] = (int)r.pitch;
    for (int i = 1; i < nd; i++) stride[i] = dat->size[i];
  }
}

char *ops_dat_get_raw_pointer(ops_dat dat, int part, ops_stencil stencil, ops_memspace *memspace) {
  (void)part;
  (void)stencil;
  return guarded([&] {
    const int ms = (memspace && *memspace == OPS_DEVICE) ? 2 : 1;
    if (memspace) *memspace = ms == 2 ? OPS_DEVICE : OPS_HOST;
    int strides[3];
    return rt().dat_get_raw_pointer(dat->index, ms, strides);
  });
}

void ops_dat_release_raw_data(ops_dat dat, int part, ops_access acc) {
  (void)part;
  guarded([&] { rt().dat_release_raw_data(dat->index, acc); });
}

void ops_dat_release_raw_data_memspace(ops_dat dat, int part, ops_access acc, ops_memspace *memspace) {
  (void)memspace;
  ops_dat_release_raw_data(dat, part, acc);
}

// ---------------------------------------------------------------------------
// Output and timers (ops/c/src/core/ops_dummy_singlenode.cpp:892-901,
// ops_lib_core.cpp:1214-1262, 1468-1626).
// ---------------------------------------------------------------------------
void ops_printf(const char *format, ...) {
  va_list ap;
  va_start(ap, format);
  print_formatted(stdout, format, ap);
  va_end(ap);
}

void ops_fprintf(FILE *stream, const char *format, ...) {
  va_list ap;
  va_start(ap, format);
  print_formatted(stream, format, ap);
  va_end(ap);
}

void ops_timers_core(double *cpu, double *et) {
  struct timeval t;
  gettimeofday(&t, nullptr);
  if (cpu) *cpu = 0.0;
  if (et) *et = (double)t.tv_sec + t.tv_usec * 1.0e-6;
}

void ops_timers(double *cpu, double *et) {
  if (Runtime::exists()) guarded([&] { Runtime::get().execute(); });
  if (Runtime::exists()) cudaStreamSynchronize(Runtime::get().stream());
  ops_timers_core(cpu, et);
}

int ops_is_root() { return opsb::Runtime::get().rank() == 0; }

// The runtime partitions across the ranks of its transport (none is set in
// a drop-in binary, so this is the single-process no-op of the reference's
// sequential and CUDA backends).
void ops_partition(const char *routine) { opsb::Runtime::get().partition(routine); }

// With diagnostics above 1 (ops_init's diags_level) the runtime times every
// kernel with CUDA events; the table lists them.
void ops_timing_output(std::ostream &stream) {
  if (!Runtime::exists()) return;
  guarded([&] {
    Runtime &r = Runtime::get();
    r.execute();
    if (r.diags() <= 1) return;
    char line[256];
    stream << "\n Kernel                                              Count    total time(sec)   GB/s\n";
    for (const auto &kv : r.kernel_times()) {
      const double s = kv.second.ms * 1e-3;
      snprintf(line, sizeof(line), " %-50s %7lld  %16.6f  %8.1f\n", kv.first.c_str(), kv.second.launches, s,
               s > 0 ? kv.second.bytes / s / 1e9 : 0.0);
      stream << line;
    }
  });
}

void ops_timing_output_stdout() { ops_timing_output(std::cout); }

void ops_diagnostic_output() {
  if (!Runtime::exists()) return;
  const Handles &h = handles();
  printf("\n OPS-B200: %zu blocks, %zu dats, %zu stencils, %zu reduction handles\n", h.blocks.size(), h.dats.size(),
         h.stencils.size(), h.reductions.size());
  for (const ops_dat_core *d : h.dats)
    printf("   dat %-20s block %-12s dim %d size %d x %d x %d\n", d->name, d->block->name, d->dim, d->size[0],
           d->size[1], d->block->dims > 2 ? d->size[2] : 1);
}

// One line per row of the dat's full extent (ops_lib_core.cpp:1272-1420
// writes the same rows with a header).
void ops_print_dat_to_txtfile_core(ops_dat dat, const char *file_name) {
  refresh_host(dat);
  FILE *f = fopen(file_name, "a");
  if (!f) {
    OPSException ex(OPS_RUNTIME_ERROR);
    ex << "cannot open " << file_name;
    throw ex;
  }
  fprintf(f, "ops_dat:  %s \n", dat->name);
  const int nx = dat->size[0];
  const size_t rows = host_bytes(dat) / ((size_t)nx * dat->elem_size);
  for (size_t r = 0; r < rows; r++) {
    for (int x = 0; x < nx; x++) {
      const char *p = dat->data + ((size_t)r * nx + x) * dat->elem_size;
      if (strcmp(dat->type, "double") == 0) fprintf(f, " %3.10lf", *(const double *)p);
      else if (strcmp(dat->type, "float") == 0) fprintf(f, " %3.10f", *(const float *)p);
      else if (strcmp(dat->type, "int") == 0) fprintf(f, " %d", *(const int *)p);
      else fprintf(f, " ?");
    }
    fprintf(f, "\n");
  }
  fclose(f);
}

void ops_print_dat_to_txtfile(ops_dat dat, const char *file_name) { ops_print_dat_to_txtfile_core(dat, file_name); }

// ops_NaNcheck (ops_lib_core.cpp:2366-2395): stops the run if a dat holds a NaN.
void ops_NaNcheck(ops_dat dat) {
  refresh_host(dat);
  if (strcmp(dat->type, "double") != 0) return;
  const double *v = reinterpret_cast<const double *>(dat->data);
  const size_t n = host_bytes(dat) / sizeof(double);
  for (size_t i = 0; i < n; i++)
    if (std::isnan(v[i])) {
      OPSException ex(OPS_RUNTIME_ERROR);
      ex << "NaN found in dat " << dat->name;
      throw ex;
    }
}

// Checkpointing (ops/c/include/ops_checkpointing.h) is out of scope: no
// checkpoint is ever restored or written, so every call reports that the run
// proceeds normally from the beginning.
bool ops_checkpointing_init(const char *filename, double interval, int options) {
  (void)filename;
  (void)interval;
  (void)options;
  return false;
}
void ops_checkpointing_initphase_done() {}
void ops_checkpointing_manual_datlist(int ndats, ops_dat *datlist) {
  (void)ndats;
  (void)datlist;
}
bool ops_checkpointing_fastfw(int nbytes, char *payload) {
  (void)nbytes;
  (void)payload;
  return false;
}
bool ops_checkpointing_manual_datlist_fastfw(int ndats, ops_dat *datlist, int nbytes, char *payload) {
  (void)ndats;
  (void)datlist;
  (void)nbytes;
  (void)payload;
  return false;
}
bool ops_checkpointing_manual_datlist_fastfw_trigger(int ndats, ops_dat *datlist, int nbytes, char *payload) {
  (void)ndats;
  (void)datlist;
  (void)nbytes;
  (void)payload;
  return false;
}
