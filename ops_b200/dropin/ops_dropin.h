// OPS-B200 drop-in layer: what code generated by the sm100a translator
// target (ops_b200/dropin/sm100a_target.py) needs besides the reference's own
// public header ops_lib_core.h, which it includes first.
//
// An OPS application keeps its sources unchanged: the reference's legacy
// translator (ops_translator_legacy/c/ops.py) rewrites each ops_par_loop into
// a call of ops_par_loop_<kernel>(name, block, dim, range, args...)
// (ops.py:731-845), and a backend target emits those functions. The sm100a
// target emits them as calls of opsb_dropin_par_loop below, which queues the
// loop on the OPS-B200 runtime with the kernel registered by the same
// generated file (a device functor made from the app's kernel function).
// ops_dropin.cu implements the reference's public API (ops_init,
// ops_decl_dat, ops_arg_dat, ops_reduction_result, ...) over that runtime with
// the reference's struct layouts (ops/c/include/ops_lib_core.h:183-552).
#pragma once

#include "runtime.h"

// Queues one loop (ops_par_loop, ops/c/include/ops_seq_v2.h:225-312): the
// reference's ops_arg records are converted to the runtime's arguments
// (dats and stencils by index, READ globals copied now, reductions by
// handle), as the reference's create_kerneldesc_and_enque does when it
// queues a loop (ops/c/src/core/ops_lazy.cpp:1403-1440).
void opsb_dropin_par_loop(const opsb::LoopInfo *loop, char const *name, ops_block block, int dim, int *range,
                          ops_arg *args, int nargs);

// The registered loop kernel named `kernel` ("<app>/<kernel name>"); throws
// if the generated file did not register it.
const opsb::LoopInfo *opsb_dropin_find_loop(const char *kernel);

// ops_decl_const / ops_update_const: the generated file copies the value to
// its own __constant__ symbol (an application and libops_b200.so each carry
// their own CUDA runtime, which knows only its own module's symbols). This
// runs the queued loops first, as the reference's lazy execution does, and
// returns the runtime's stream for the copy; opsb_dropin_const_done waits for
// it and reports a failed copy as an OPSException.
cudaStream_t opsb_dropin_const_begin();
void opsb_dropin_const_done(cudaError_t copy_status, const char *name);
