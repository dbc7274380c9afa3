// Device-side building blocks of the OPS-B200 loop backend.
//
// An OPS parallel loop (ops_par_loop, ops/c/include/ops_seq_v2.h:225-292 is
// the semantic reference) applies a per-point kernel over an index range;
// the kernel reaches neighbouring points of each dat through an accessor
// (ACC<T>, ops/c/include/ops_lib_core.h:1357-2038) and receives global
// arguments (ops_arg_gbl), reduction targets (ops_arg_reduce) and the
// point's index (ops_arg_idx) through plain pointers.
//
// Here each loop kernel is a functor with a __device__ operator() taking the
// same parameter list as the OPS kernel; ACC2/ACC3 play the role of ACC<T>.
// exec_loop<K> (below) turns the functor into a grid: x is the fastest,
// coalesced dimension, each thread walks several rows, reductions are folded
// per thread, per warp (shuffles), per block (shared memory) and finally
// across blocks by the last block to finish, in a fixed order, so results do
// not depend on scheduling.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <float.h>
#include <limits.h>
#include <utility>
#include <type_traits>

#define OPSB_MAX_ARGS 24
#define OPSB_MAX_RED_DIM 12
#define OPSB_MAX_REDUCE_ARGS 8

namespace opsb {

enum ArgKind { ARG_GBL = 0, ARG_DAT = 1, ARG_IDX = 2, ARG_REDUCE = 3 };
// Access modes keep the reference's numbering (ops/c/include/ops_lib_core.h:84-89).
enum Access { ACC_READ = 0, ACC_WRITE = 1, ACC_RW = 2, ACC_INC = 3, ACC_MIN = 4, ACC_MAX = 5 };

// The reference's min/max/sign macros (ops/c/include/ops_lib_core.h:559-571),
// restated as functions with the same comparison order so that ties, signed
// zeros and NaNs resolve exactly as on the CPU.
template <class T> __host__ __device__ __forceinline__ T op_min(T a, T b) { return (a < b) ? a : b; }
template <class T> __host__ __device__ __forceinline__ T op_max(T a, T b) { return (a > b) ? a : b; }
__host__ __device__ __forceinline__ double op_sign(double a, double b) { return (b < 0.0) ? (a * (-1)) : a; }
// a / b, with the same IEEE result for every input. When a is a zero and b
// finite and nonzero the quotient is the zero of sign(a) xor sign(b), which
// a * b also gives; the product then replaces the correctly rounded
// division, whose general path is far longer. In the quiescent regions of
// the hydro kernels most of these numerators (velocity differences,
// fluxes, viscosity) are exactly zero; CloverLeaf 2D viscosity_kernel went
// from 0.43 to 0.18 ms per launch at 3840^2.
__device__ __forceinline__ double qdiv(double a, double b) {
  if (a == 0.0 && b != 0.0 && isfinite(b)) return a * b;
  return a / b;
}
// a / b, with the same IEEE result for every input: equal finite nonzero
// operands give exactly 1 without the division (the cell-width ratios of a
// uniform mesh).
__device__ __forceinline__ double qratio(double a, double b) {
  if (a == b && b != 0.0 && isfinite(b)) return 1.0;
  return a / b;
}

// 2D accessor: p points at the current point; (i, j) is a stencil offset.
// As in the reference's ACC<T> (ops/c/include/ops_lib_core.h:1525-1556) an
// offset is i + j * (row pitch) whatever the stencil's stride: a dat that is
// one point wide along a dimension is only ever offset along the other.
// `coherent` selects how a read-only view loads: 0 through the non-coherent
// read-only path (data no thread writes during the kernel: every argument of
// a single loop kernel, where the flag is the constant 0 and the test folds
// away), 1 with ordinary loads through a generic address (fused chain
// kernels, whose views may point into shared-memory tiles or at data other
// phases of the same kernel write).
template <class T>
struct ACC2 {
  using value_type = T;
  T *p;
  int sy;
  int coherent;
  ACC2() = default;
  __device__ __forceinline__ ACC2(T *p_, int sy_) : p(p_), sy(sy_), coherent(0) {}
  __device__ __forceinline__ ACC2(T *p_, int sy_, int coh) : p(p_), sy(sy_), coherent(coh) {}
  __device__ __forceinline__ T &operator()(int i, int j) { return p[i + j * sy]; }
  // Read-only view (the kernel's const ACC<T>& arguments).
  __device__ __forceinline__ T operator()(int i, int j) const {
    return coherent ? p[i + j * sy] : __ldg(p + (i + j * sy));
  }
};

// 3D accessor.
template <class T>
struct ACC3 {
  T *p;
  int sy, sz;
  ACC3() = default;
  __device__ __forceinline__ ACC3(T *p_, int sy_, int sz_) : p(p_), sy(sy_), sz(sz_) {}
  __device__ __forceinline__ T &operator()(int i, int j, int k) { return p[i + j * sy + (long long)k * sz]; }
  __device__ __forceinline__ T operator()(int i, int j, int k) const {
    return __ldg(p + (i + j * sy + (long long)k * sz));
  }
};

// Reduction target of a kernel (the reference passes a T*): a thread-local
// accumulator of N components kept in registers; *r and r[i] read like the
// reference's pointer.
template <class T, int N = 1>
struct RED {
  T v[N];
  __device__ __forceinline__ T &operator*() { return v[0]; }
  __device__ __forceinline__ T &operator[](int i) { return v[i]; }
};

// The point's index (ops_arg_idx; the reference passes const int*).
struct IDX {
  int v[3];
  __device__ __forceinline__ int operator[](int i) const { return v[i]; }
};

// One loop argument as the device sees it.
struct ArgView {
  char *ptr;        // DAT: logical origin of the dat; GBL: device copy; REDUCE: handle slot
  int sx, sy, sz;   // element strides of the point's base (0 where the stencil does not stride)
  int ay, az;       // accessor strides: row pitch and plane size of the dat
  int kind;         // ArgKind
  int acc;          // Access
  int dim;          // components (reduction width for REDUCE)
  int red_index;    // REDUCE: index among this loop's reduction args
  int first;        // REDUCE: 1 when the handle starts from the identity in this loop
  int mg;           // DAT: 0 plain, 1 prolong, 2 restrict stencil (multigrid)
  int ms[3];        // DAT: the multigrid stencil's stride per dimension
};

struct LoopParams {
  int start[3], end[3];
  int ndim;
  int nargs;
  int nred;           // number of REDUCE args
  int rows_per_iter;  // unused by exec_loop, kept for fused kernels
  char *red_scratch;  // per-block partials: [red_index][block][OPSB_MAX_RED_DIM] x 8 bytes
  unsigned int *red_counter;  // blocks-done counter, reset to 0 by the last block
  ArgView a[OPSB_MAX_ARGS];
};

// ----------------------------------------------------------------------------
// Reduction identities and combine, by element type and access mode
// (zero / +max / -max as ops/c/include/ops_internal2.h:67-97 defines them).
// ----------------------------------------------------------------------------
template <class T> struct RedTraits;
template <> struct RedTraits<double> { __device__ static double big() { return DBL_MAX; } };
template <> struct RedTraits<float> { __device__ static float big() { return FLT_MAX; } };
template <> struct RedTraits<int> { __device__ static int big() { return INT_MAX; } };
template <> struct RedTraits<long long> { __device__ static long long big() { return LLONG_MAX; } };

template <class T>
__device__ __forceinline__ T red_identity(int acc) {
  if (acc == ACC_MIN) return RedTraits<T>::big();
  if (acc == ACC_MAX) return -RedTraits<T>::big();
  return T(0);
}
template <class T>
__device__ __forceinline__ T red_combine(int acc, T a, T b) {
  if (acc == ACC_MIN) return op_min(a, b);
  if (acc == ACC_MAX) return op_max(a, b);
  return a + b;
}

template <class T>
__device__ __forceinline__ T shfl_down(T v, int o) { return __shfl_down_sync(0xffffffffu, v, o); }

// Block-wide reduction of one value; result valid in thread 0.
// smem must hold one T per warp.
template <class T>
__device__ __forceinline__ T block_reduce(T v, int acc, T *smem) {
  const int lane = threadIdx.x & 31;
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  const int warp = tid >> 5;
  const int nwarps = (blockDim.x * blockDim.y + 31) >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = red_combine(acc, v, shfl_down(v, o));
  __syncthreads();
  if (lane == 0) smem[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = (lane < nwarps) ? smem[lane] : red_identity<T>(acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = red_combine(acc, v, shfl_down(v, o));
  }
  return v;
}

// ----------------------------------------------------------------------------
// Per-parameter storage: how each kernel parameter is produced from an arg.
// ----------------------------------------------------------------------------
template <class P> struct Slot;

template <class T>
struct Slot<ACC2<T>> {
  ACC2<T> acc;
  __device__ __forceinline__ void init(const ArgView &) {}
  __device__ __forceinline__ ACC2<T> &at(const ArgView &a, int x, int y, int) {
    acc = ACC2<T>(reinterpret_cast<T *>(a.ptr) + (x * a.sx + y * a.sy), a.ay);
    return acc;
  }
  template <class S> __device__ __forceinline__ void finish(const ArgView &, const LoopParams &, S *, int) {}
};

template <class T>
struct Slot<ACC3<T>> {
  ACC3<T> acc;
  __device__ __forceinline__ void init(const ArgView &) {}
  __device__ __forceinline__ ACC3<T> &at(const ArgView &a, int x, int y, int z) {
    acc = ACC3<T>(reinterpret_cast<T *>(a.ptr) + (x * a.sx + y * a.sy + (long long)z * a.sz), a.ay, a.az);
    return acc;
  }
  template <class S> __device__ __forceinline__ void finish(const ArgView &, const LoopParams &, S *, int) {}
};

template <class T, int N>
struct Slot<RED<T, N>> {
  RED<T, N> r;
  __device__ __forceinline__ void init(const ArgView &a) {
#pragma unroll
    for (int d = 0; d < N; d++) r.v[d] = red_identity<T>(a.acc);
  }
  __device__ __forceinline__ RED<T, N> &at(const ArgView &, int, int, int) { return r; }
  // Fold this thread's partial into the block's and store the block partial.
  __device__ void finish(const ArgView &a, const LoopParams &lp, T *smem, int nblocks) {
    const int bid = blockIdx.x + blockIdx.y * gridDim.x;
    T *part = reinterpret_cast<T *>(lp.red_scratch) + ((size_t)a.red_index * nblocks + bid) * OPSB_MAX_RED_DIM;
#pragma unroll
    for (int d = 0; d < N; d++) {
      T v = block_reduce<T>(r.v[d], a.acc, smem);
      if (threadIdx.x == 0 && threadIdx.y == 0 && d < a.dim) part[d] = v;
    }
  }
};

template <>
struct Slot<IDX> {
  IDX i;
  __device__ __forceinline__ void init(const ArgView &) {}
  __device__ __forceinline__ IDX &at(const ArgView &, int x, int y, int z) {
    i.v[0] = x; i.v[1] = y; i.v[2] = z;
    return i;
  }
};

// Multigrid stencils address a dat of another resolution: a restrict
// stencil reads the fine dat at x * stride, a prolong stencil the coarse dat
// at floor(x / stride), stencil offsets added after (the addressing the
// reference generates for them, ops_translator_legacy/c/ops_gen_mpi_lazy.py:283-315,
// for non-negative loop starts).
__device__ __forceinline__ int mg_index(int x, int mode, int s) {
  if (mode == 2) return x * s;
  if (mode == 1) return x >= 0 ? x / s : -((s - 1 - x) / s);
  return x;
}
template <class P> struct is_accessor_slot : std::false_type {};
template <class T> struct is_accessor_slot<ACC2<T>> : std::true_type {};
template <class T> struct is_accessor_slot<ACC3<T>> : std::true_type {};

// Pointer parameters are globals (ops_arg_gbl): READ as const T*, RW as T*.
template <class T>
struct Slot<T *> {
  __device__ __forceinline__ void init(const ArgView &) {}
  __device__ __forceinline__ T *at(const ArgView &a, int, int, int) { return reinterpret_cast<T *>(a.ptr); }
};

// Minimal tuple of slots (device code, no std::tuple).
template <size_t I, class T> struct Leaf { T v; };
template <class Seq, class... T> struct SlotTuple;
template <size_t... I, class... T>
struct SlotTuple<std::index_sequence<I...>, T...> : Leaf<I, T>... {};
template <size_t I, class T> __device__ __forceinline__ T &get_leaf(Leaf<I, T> &l) { return l.v; }

// Reduction element type of a parameter (void when it cannot reduce).
template <class P> struct RedElem { using type = void; };
template <class T, int N> struct RedElem<RED<T, N>> { using type = T; };

// Combine the per-block partials of every reduction arg (last block only).
template <class T>
__device__ void finish_grid_reduction(const ArgView &a, const LoopParams &lp, int nblocks, T *smem) {
  T *part = reinterpret_cast<T *>(lp.red_scratch) + (size_t)a.red_index * nblocks * OPSB_MAX_RED_DIM;
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  const int nthr = blockDim.x * blockDim.y;
  T *slot = reinterpret_cast<T *>(a.ptr);
  for (int d = 0; d < a.dim; d++) {
    T v = red_identity<T>(a.acc);
    for (int b = tid; b < nblocks; b += nthr) v = red_combine(a.acc, v, part[(size_t)b * OPSB_MAX_RED_DIM + d]);
    v = block_reduce<T>(v, a.acc, smem);
    if (tid == 0) slot[d] = a.first ? v : red_combine(a.acc, slot[d], v);
  }
}

template <class A> struct is_acc2 : std::false_type {};
template <class T> struct is_acc2<ACC2<T>> : std::true_type {};

// Kernels that may be given restrict/prolong stencils state `mgrid = true`
// (their accessors then map the point's index per argument).
template <class K, class = void> struct LoopMgridOk { static constexpr bool value = false; };
template <class K> struct LoopMgridOk<K, std::void_t<decltype(K::mgrid)>> {
  static constexpr bool value = K::mgrid;
};

template <class K, class Sig> struct Exec;

template <class K, class C, class... P>
struct Exec<K, void (C::*)(P...) const> {
  using Seq = std::index_sequence_for<P...>;
  using Tup = SlotTuple<Seq, Slot<std::decay_t<P>>...>;

  template <size_t... I>
  __device__ static __forceinline__ void init_all(Tup &t, const LoopParams &lp, std::index_sequence<I...>) {
    (get_leaf<I, Slot<std::decay_t<P>>>(t).init(lp.a[I]), ...);
  }
  template <size_t... I>
  __device__ static __forceinline__ void call(const K &k, Tup &t, const LoopParams &lp, int x, int y, int z,
                                              std::index_sequence<I...>) {
    k(slot_at<I>(t, lp, x, y, z)...);
  }
  template <size_t I>
  __device__ static __forceinline__ decltype(auto) slot_at(Tup &t, const LoopParams &lp, int x, int y, int z) {
    using PT = std::decay_t<std::tuple_element_t<I, std::tuple<P...>>>;
    auto &sl = get_leaf<I, Slot<PT>>(t);
    if constexpr (LoopMgridOk<K>::value && is_accessor_slot<PT>::value) {
      const ArgView &a = lp.a[I];
      return sl.at(a, mg_index(x, a.mg, a.ms[0]), mg_index(y, a.mg, a.ms[1]), mg_index(z, a.mg, a.ms[2]));
    } else {
      return sl.at(lp.a[I], x, y, z);
    }
  }
  // L2 prefetch hint for the centre point of every read-only accessor at
  // (x, y): a thread asks for its next row before working on this one.
  template <size_t... I>
  __device__ static __forceinline__ void touch_all(const LoopParams &lp, int x, int y, std::index_sequence<I...>) {
    (touch_one<I>(lp, x, y), ...);
  }
  template <size_t I>
  __device__ static __forceinline__ void touch_one(const LoopParams &lp, int x, int y) {
    using RP = std::remove_reference_t<std::tuple_element_t<I, std::tuple<P...>>>;
    if constexpr (std::is_const<RP>::value && is_acc2<std::remove_const_t<RP>>::value) {
      using T = typename std::remove_const_t<RP>::value_type;
      const ArgView &a = lp.a[I];
      const T *p = reinterpret_cast<const T *>(a.ptr) + (x * a.sx + y * a.sy);
      asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
    }
  }
  template <size_t... I>
  __device__ static __forceinline__ void finish_all(Tup &t, const LoopParams &lp, double *smem, int nblocks,
                                                    std::index_sequence<I...>) {
    (finish_one<I>(t, lp, smem, nblocks), ...);
  }
  template <size_t I>
  __device__ static __forceinline__ void finish_one(Tup &t, const LoopParams &lp, double *smem, int nblocks) {
    using PT = std::decay_t<std::tuple_element_t<I, std::tuple<P...>>>;
    using RT = typename RedElem<PT>::type;
    if constexpr (!std::is_void<RT>::value) {
      get_leaf<I, Slot<PT>>(t).finish(lp.a[I], lp, reinterpret_cast<RT *>(smem), nblocks);
    }
  }
  template <size_t... I>
  __device__ static __forceinline__ void grid_finish_all(const LoopParams &lp, double *smem, int nblocks,
                                                         std::index_sequence<I...>) {
    (grid_finish_one<I>(lp, smem, nblocks), ...);
  }
  template <size_t I>
  __device__ static __forceinline__ void grid_finish_one(const LoopParams &lp, double *smem, int nblocks) {
    using PT = std::decay_t<std::tuple_element_t<I, std::tuple<P...>>>;
    using RT = typename RedElem<PT>::type;
    if constexpr (!std::is_void<RT>::value) {
      finish_grid_reduction<RT>(lp.a[I], lp, nblocks, reinterpret_cast<RT *>(smem));
    }
  }
};

// Resident 256-thread CTAs per SM the register allocation must allow: 8
// (a full SM, at most 32 registers a thread) unless a kernel states
// `min_blocks`. The loops are latency-bound streams whose loads cannot be
// hoisted over the previous point's stores, so the bytes in flight per SM
// grow with the resident threads: occupancy is worth a few spills.
#ifndef OPSB_MIN_BLOCKS
#define OPSB_MIN_BLOCKS 8
#endif
template <class K, class = void> struct LoopMinBlocks { static constexpr int value = OPSB_MIN_BLOCKS; };
template <class K> struct LoopMinBlocks<K, std::void_t<decltype(K::min_blocks)>> {
  static constexpr int value = K::min_blocks;
};

// Rows a thread keeps in flight in the 2D row loop (memory-level
// parallelism of the streaming loops); a kernel may state `row_unroll`.
#ifndef OPSB_ROW_UNROLL
#define OPSB_ROW_UNROLL 2
#endif
template <class K, class = void> struct LoopRowUnroll { static constexpr int value = OPSB_ROW_UNROLL; };
template <class K> struct LoopRowUnroll<K, std::void_t<decltype(K::row_unroll)>> {
  static constexpr int value = K::row_unroll;
};

// Next-row prefetch hints (Exec::touch_all) in the 2D row loop: they help
// the loops whose reads are few and far between stores and slow down the
// rest, so a kernel opts in with `touch_next_row` (measured per kernel).
template <class K, class = void> struct LoopTouch { static constexpr bool value = false; };
template <class K> struct LoopTouch<K, std::void_t<decltype(K::touch_next_row)>> {
  static constexpr bool value = K::touch_next_row;
};

// The generic loop kernel. blockDim = (BX, BY); blocks tile x exactly and
// stride over the remaining (y, z) rows.
template <class K>
__global__ void __launch_bounds__(256, LoopMinBlocks<K>::value) exec_loop(const __grid_constant__ LoopParams lp) {
  using E = Exec<K, decltype(&K::operator())>;
  typename E::Tup t;
  E::init_all(t, lp, typename E::Seq{});
  const K k{};
  const int x = lp.start[0] + blockIdx.x * blockDim.x + threadIdx.x;
  const int ny = lp.end[1] - lp.start[1];
  const int nz = lp.end[2] - lp.start[2];
  const long long nrows = (long long)ny * nz;
  if (x < lp.end[0]) {
    if (nz == 1) {
      constexpr int kUnroll = LoopRowUnroll<K>::value;
#pragma unroll (kUnroll)
      for (int y = lp.start[1] + blockIdx.y * blockDim.y + threadIdx.y; y < lp.end[1]; y += gridDim.y * blockDim.y) {
        if constexpr (LoopTouch<K>::value)
          if (y + (int)(gridDim.y * blockDim.y) < lp.end[1])
            E::touch_all(lp, x, y + gridDim.y * blockDim.y, typename E::Seq{});
        E::call(k, t, lp, x, y, lp.start[2], typename E::Seq{});
      }
    } else {
      for (long long r = (long long)blockIdx.y * blockDim.y + threadIdx.y; r < nrows;
           r += (long long)gridDim.y * blockDim.y) {
        const int y = lp.start[1] + (int)(r % ny);
        const int z = lp.start[2] + (int)(r / ny);
        E::call(k, t, lp, x, y, z, typename E::Seq{});
      }
    }
  }
  if (lp.nred == 0) return;
  __shared__ double smem[32];
  const int nblocks = gridDim.x * gridDim.y;
  E::finish_all(t, lp, smem, nblocks, typename E::Seq{});
  __shared__ int last;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    __threadfence();
    unsigned int done = atomicAdd(lp.red_counter, 1u);
    last = (done == (unsigned int)(nblocks - 1));
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  E::grid_finish_all(lp, smem, nblocks, typename E::Seq{});
  if (threadIdx.x == 0 && threadIdx.y == 0) *lp.red_counter = 0u;
}

// Several queued loops of one kernel, each over its own block or range (the
// uneven domains of a multi-block application), in one launch: item i owns
// the CTAs [first, first + gx * gy) of the linear grid and runs them as
// exec_loop's (gx, gy) grid would. Loops with reductions are not batched.
struct ListItem {
  int gx, gy;
  long long first;
};

template <class K>
__global__ void __launch_bounds__(256, LoopMinBlocks<K>::value)
    exec_loop_list(const LoopParams *__restrict__ items, const ListItem *__restrict__ grids, int nitems) {
  using E = Exec<K, decltype(&K::operator())>;
  const long long b = blockIdx.x;
  int lo = 0, hi = nitems - 1;  // last item whose first CTA is <= b
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (grids[mid].first <= b) lo = mid;
    else hi = mid - 1;
  }
  const LoopParams &lp = items[lo];
  const ListItem g = grids[lo];
  const int local = (int)(b - g.first);
  const int bx = local % g.gx, by = local / g.gx;
  typename E::Tup t;
  E::init_all(t, lp, typename E::Seq{});
  const K k{};
  const int x = lp.start[0] + bx * blockDim.x + threadIdx.x;
  const int ny = lp.end[1] - lp.start[1];
  const int nz = lp.end[2] - lp.start[2];
  const long long nrows = (long long)ny * nz;
  if (x >= lp.end[0]) return;
  const int ystep = g.gy * blockDim.y;
  if (nz == 1) {
    for (int y = lp.start[1] + by * blockDim.y + threadIdx.y; y < lp.end[1]; y += ystep)
      E::call(k, t, lp, x, y, lp.start[2], typename E::Seq{});
  } else {
    for (long long r = (long long)by * blockDim.y + threadIdx.y; r < nrows; r += ystep) {
      const int y = lp.start[1] + (int)(r % ny);
      const int z = lp.start[2] + (int)(r / ny);
      E::call(k, t, lp, x, y, z, typename E::Seq{});
    }
  }
}

// Host-side description of a kernel's parameter list, used to validate args
// at enqueue time: 'A' accessor, 'R' reduction (ndim = width), 'I' index,
// 'p' non-const pointer, 'c' const pointer; elem is the element size in bytes.
struct ParamInfo { char cls; int elem; int ndim; };

template <class P> struct ParamDesc;
template <class T> struct ParamDesc<ACC2<T>> { static ParamInfo get() { return {'A', (int)sizeof(T), 2}; } };
template <class T> struct ParamDesc<ACC3<T>> { static ParamInfo get() { return {'A', (int)sizeof(T), 3}; } };
template <class T> struct ParamDesc<T *> { static ParamInfo get() { return {'p', (int)sizeof(T), 0}; } };
template <class T, int N> struct ParamDesc<RED<T, N>> { static ParamInfo get() { return {'R', (int)sizeof(T), N}; } };
template <> struct ParamDesc<IDX> { static ParamInfo get() { return {'I', 4, 0}; } };
template <class T> struct ParamDesc<const T *> { static ParamInfo get() { return {'c', (int)sizeof(T), 0}; } };

template <class Sig> struct SigInfo;
template <class C, class... P>
struct SigInfo<void (C::*)(P...) const> {
  static constexpr int n = sizeof...(P);
  static void fill(ParamInfo *out) {
    ParamInfo tmp[] = {ParamDesc<std::decay_t<P>>::get()..., ParamInfo{0, 0, 0}};
    for (int i = 0; i < (int)sizeof...(P); i++) out[i] = tmp[i];
  }
};

}  // namespace opsb
