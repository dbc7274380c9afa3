// Device side of loop-chain fusion (see fusion.h for the plan and the rules
// that bind each dat).
//
// fused_chain_kernel<G> runs a chain of loops whose compute kernels are
// functors of the group G (a compile-time list; a loop names its functor by
// index). One CTA of 256 threads walks tiles of the grid: it stages the
// tiles the plan asks for into shared memory, runs every loop of the chain
// over its region (the tile's core grown by the loop's halo depths, cut to
// the loop's range) with a barrier between loops, writes the shared-memory
// tiles' results back, and moves to its next tile. Min/max reductions are
// folded per thread over all its points, then per block and across blocks
// by the last block to finish, as in exec_loop.
#pragma once
#include <utility>

#include "fusion.h"
#include "ops_b200_device.cuh"

namespace opsb {
namespace fuse {

struct TileCtx {
  const FPlan *P;
  double *sm;
  // Write sink for masked points: this thread's own kScratch doubles, one
  // cell per argument (at +16 + its index in the loop, so that stencil
  // offsets of up to 16 stay inside). Per thread and per argument, because
  // kernels read back what they wrote through arguments declared
  // write-only (CloverLeaf's accelerate_kernel reads stepbymass after
  // setting it; advec_cell_kernel4 reads pre_mass, post_mass and advec_vol).
  double *scratch;
  double *racc;      // per-thread reduction accumulators
  int cx0, cy0, cx1, cy1;
};

// Per-point work is kept free of memory the kernels' stores could alias:
// every slot copies what it needs from the plan (global memory) into its own
// members when a phase starts, and writes reduction partials back when it
// ends, so a point costs only its address arithmetic and the kernel's own
// loads and stores.
template <class P> struct FSlot;

// An accessor argument: where its point (x, y) lives is resolved once per
// phase (a shared-memory tile, or the dat in HBM), so that a point costs
// one multiply-add per argument. Views are always coherent generic loads:
// they may point into shared-memory tiles or at data other phases write.
template <class T>
struct FSlot<ACC2<T>> {
  ACC2<T> acc;
  T *base;       // address of logical (0, 0) in the bound storage (may lie outside it)
  int sx, sy, ay;
  bool masked;
  T *sink;
  __device__ __forceinline__ void init(const TileCtx &c, const FArg &a) {
    if (a.mode == M_TILE) {
      const FBuf &b = c.P->B[a.buf];
      const long long o = (long long)b.off - (c.cx0 - b.hx0) - (long long)(c.cy0 - b.hy0) * b.pitch;
      base = reinterpret_cast<T *>(c.sm) + o;
      sx = 1;
      sy = ay = b.pitch;
    } else {
      base = reinterpret_cast<T *>(a.ptr);
      sx = a.sx;
      sy = a.sy;
      ay = a.ay;
    }
    masked = a.mode == M_RW && a.masked;
    sink = reinterpret_cast<T *>(c.scratch + 16 + a.slot);
  }
  __device__ __forceinline__ ACC2<T> &at(int x, int y, bool core) {
    acc = (masked && !core) ? ACC2<T>(sink, 0, 1) : ACC2<T>(base + (x * sx + y * sy), ay, 1);
    return acc;
  }
  __device__ __forceinline__ void done(bool) {}
  __device__ __forceinline__ void fini(const TileCtx &, const FArg &) {}
};

template <class T, int N>
struct FSlot<RED<T, N>> {
  static_assert(N == 1, "fused chains take one-component reductions");
  RED<T, N> r;
  T part, ident;  // this thread's partial over the core's points; the identity
  __device__ __forceinline__ void init(const TileCtx &c, const FArg &a) {
    part = (T)c.racc[a.red];
    ident = red_identity<T>(c.P->red[a.red].acc);
  }
  __device__ __forceinline__ RED<T, N> &at(int, int, bool core) {
    r.v[0] = core ? part : ident;
    return r;
  }
  __device__ __forceinline__ void done(bool core) {
    if (core) part = r.v[0];
  }
  __device__ __forceinline__ void fini(const TileCtx &c, const FArg &a) { c.racc[a.red] = (double)part; }
};

template <>
struct FSlot<IDX> {
  IDX i;
  __device__ __forceinline__ void init(const TileCtx &, const FArg &) {}
  __device__ __forceinline__ IDX &at(int x, int y, bool) {
    i.v[0] = x;
    i.v[1] = y;
    i.v[2] = 0;
    return i;
  }
  __device__ __forceinline__ void done(bool) {}
  __device__ __forceinline__ void fini(const TileCtx &, const FArg &) {}
};

template <class T>
struct FSlot<T *> {
  T *p;
  __device__ __forceinline__ void init(const TileCtx &, const FArg &a) { p = reinterpret_cast<T *>(a.ptr); }
  __device__ __forceinline__ T *at(int, int, bool) { return p; }
  __device__ __forceinline__ void done(bool) {}
  __device__ __forceinline__ void fini(const TileCtx &, const FArg &) {}
};

template <class K, class Sig> struct FusedCall;
template <class K, class C, class... P>
struct FusedCall<K, void (C::*)(P...) const> {
  using Seq = std::index_sequence_for<P...>;
  using Tup = SlotTuple<Seq, FSlot<std::decay_t<P>>...>;

  template <size_t... I>
  __device__ static __forceinline__ void init_all(Tup &t, const TileCtx &c, const FArg *a, std::index_sequence<I...>) {
    (get_leaf<I, FSlot<std::decay_t<P>>>(t).init(c, a[I]), ...);
  }
  template <size_t... I>
  __device__ static __forceinline__ void fini_all(Tup &t, const TileCtx &c, const FArg *a, std::index_sequence<I...>) {
    (get_leaf<I, FSlot<std::decay_t<P>>>(t).fini(c, a[I]), ...);
  }
  template <size_t... I>
  __device__ static __forceinline__ void point(const K &k, Tup &t, int x, int y, bool core,
                                               std::index_sequence<I...>) {
    k(get_leaf<I, FSlot<std::decay_t<P>>>(t).at(x, y, core)...);
    (get_leaf<I, FSlot<std::decay_t<P>>>(t).done(core), ...);
  }

  // All points of the loop's region in this tile; consecutive threads take
  // consecutive x so that HBM accesses coalesce. A thread steps through the
  // region by a fixed (dx, dy) instead of dividing its flat index per point.
  __device__ static __forceinline__ void phase(const TileCtx &c, const FLoop &L, int rx0, int rx1, int ry0,
                                               int ry1) {
    const K k{};
    Tup t;
    const FArg *a = c.P->A + L.arg0;
    init_all(t, c, a, Seq{});
    const int w = rx1 - rx0;
    const int cx0 = c.cx0, cx1 = c.cx1, cy0 = c.cy0, cy1 = c.cy1;
    const int dy = kThreads / w, dx = kThreads - dy * w;
    int y = ry0 + (int)threadIdx.x / w;
    int x = rx0 + ((int)threadIdx.x - (y - ry0) * w);
    for (; y < ry1;) {
      const bool core = x >= cx0 && x < cx1 && y >= cy0 && y < cy1;
      point(k, t, x, y, core, Seq{});
      x += dx;
      y += dy;
      if (x >= rx1) {
        x -= w;
        y++;
      }
    }
    fini_all(t, c, a, Seq{});
  }
};

// A compile-time list of loop functors; dispatch by index.
template <int MinBlocks, class... K>
struct Group {
  static constexpr int size = sizeof...(K);
  static constexpr int min_blocks = MinBlocks;
  template <int I, class First, class... Rest>
  __device__ static __forceinline__ void run_at(int kid, const TileCtx &c, const FLoop &L, int rx0, int rx1,
                                                int ry0, int ry1) {
    if (kid == I) {
      FusedCall<First, decltype(&First::operator())>::phase(c, L, rx0, rx1, ry0, ry1);
      return;
    }
    if constexpr (sizeof...(Rest) > 0) run_at<I + 1, Rest...>(kid, c, L, rx0, rx1, ry0, ry1);
  }
  __device__ static void run(int kid, const TileCtx &c, const FLoop &L, int rx0, int rx1, int ry0, int ry1) {
    run_at<0, K...>(kid, c, L, rx0, rx1, ry0, ry1);
  }
};

// Address of (x, y) of an argument bound RO/RW/TILE (copy loops).
__device__ __forceinline__ double *fused_addr(const TileCtx &c, const FArg &a, int x, int y) {
  if (a.mode == M_TILE) {
    const FBuf &b = c.P->B[a.buf];
    return c.sm + b.off + (x - (c.cx0 - b.hx0)) + (y - (c.cy0 - b.hy0)) * b.pitch;
  }
  return reinterpret_cast<double *>(a.ptr) + (x * a.sx + y * a.sy);
}

// A boundary copy loop: each listed field copies (or negates) the value at
// the mirror point (x+ox, y+oy). Points outside the core write only fields
// bound to shared-memory tiles.
__device__ inline void copy_phase(const TileCtx &c, const FLoop &L, int rx0, int rx1, int ry0, int ry1) {
  const FArg *a = c.P->A + L.arg0;
  const int w = rx1 - rx0;
  const int cx0 = c.cx0, cx1 = c.cx1, cy0 = c.cy0, cy1 = c.cy1;
  const int ox = L.cp_ox, oy = L.cp_oy, nf = L.cp_n;
  const bool neg = L.cp_neg != 0;
  const int dy = kThreads / w, dx = kThreads - dy * w;
  // one field at a time: its address arithmetic is read from the plan once
  for (int f = 0; f < nf; f++) {
    const FArg &fa = a[L.cp_arg[f]];
    const bool tile = fa.mode == M_TILE;
    double *const o = fused_addr(c, fa, 0, 0);
    int sx = 1, sy;
    if (tile) {
      sy = c.P->B[fa.buf].pitch;
    } else {
      sx = fa.sx;
      sy = fa.sy;
    }
    const int moff = ox * sx + oy * sy;
    int y = ry0 + (int)threadIdx.x / w;
    int x = rx0 + ((int)threadIdx.x - (y - ry0) * w);
    for (; y < ry1;) {
      if (tile || (x >= cx0 && x < cx1 && y >= cy0 && y < cy1)) {
        double *q = o + (x * sx + y * sy);
        const double v = q[moff];
        *q = neg ? -v : v;
      }
      x += dx;
      y += dy;
      if (x >= rx1) {
        x -= w;
        y++;
      }
    }
  }
}

// G::min_blocks: CTAs per SM the register allocation must allow (the
// group's functors decide how many registers that leaves).
template <class G>
__global__ void __launch_bounds__(kThreads, G::min_blocks) fused_chain_kernel(const FPlan *__restrict__ P) {
  extern __shared__ double sm_all[];
  double scratch[kScratch];
  __shared__ double red_smem[32];
  __shared__ int last;
  double racc[kMaxRed];
  const int nred = P->nred;
  for (int r = 0; r < kMaxRed; r++) racc[r] = r < nred ? red_identity<double>(P->red[r].acc) : 0.0;
  double *sm = sm_all + kGuard;
  // guards: zero once
  for (int i = threadIdx.x; i < kGuard; i += kThreads) {
    sm_all[i] = 0.0;
    sm_all[P->smem_doubles - kGuard + i] = 0.0;
  }
  TileCtx c;
  c.P = P;
  c.sm = sm;
  c.scratch = scratch;
  c.racc = racc;
  const int TX = P->TX, TY = P->TY, ntx = P->ntx;
  const int ntiles = ntx * P->nty;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int ty = t / ntx;
    c.cx0 = P->gx0 + (t - ty * ntx) * TX;
    c.cy0 = P->gy0 + ty * TY;
    c.cx1 = c.cx0 + TX;
    c.cy1 = c.cy0 + TY;
    // stage the tiles that hold values from before the chain
    for (int b = 0; b < P->nbufs; b++) {
      const FBuf &B = P->B[b];
      if (!B.src) continue;
      const int x0 = max(c.cx0 - B.hx0, B.ax0), x1 = min(c.cx1 + B.hx1, B.ax1);
      const int y0 = max(c.cy0 - B.hy0, B.ay0), y1 = min(c.cy1 + B.hy1, B.ay1);
      const int w = x1 - x0;
      if (w <= 0 || y1 <= y0) continue;
      const double *src = reinterpret_cast<const double *>(B.src);
      double *dst = sm + B.off + (x0 - (c.cx0 - B.hx0)) + (y0 - (c.cy0 - B.hy0)) * B.pitch;
      src += x0 + (long long)y0 * B.ay;
      // asynchronous copies (cp.async, 8 bytes each): every tile's loads are
      // in flight at once instead of one dependent load per thread at a time
      const int dy = kThreads / w, dx = kThreads - dy * w;
      int yy = (int)threadIdx.x / w;
      int xx = (int)threadIdx.x - yy * w;
      for (; yy < y1 - y0;) {
        const unsigned int s_addr = (unsigned int)__cvta_generic_to_shared(dst + xx + yy * B.pitch);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s_addr), "l"(src + xx + (long long)yy * B.ay)
                     : "memory");
        xx += dx;
        yy += dy;
        if (xx >= w) {
          xx -= w;
          yy++;
        }
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    for (int l = 0; l < P->nloops; l++) {
      const FLoop &L = P->L[l];
      const int rx0 = max(L.x0, c.cx0 - L.ex0), rx1 = min(L.x1, c.cx1 + L.ex1);
      const int ry0 = max(L.y0, c.cy0 - L.ey0), ry1 = min(L.y1, c.cy1 + L.ey1);
      if (rx0 >= rx1 || ry0 >= ry1) continue;  // the same for every thread of the block
      if (L.kid < 0)
        copy_phase(c, L, rx0, rx1, ry0, ry1);
      else
        G::run(L.kid, c, L, rx0, rx1, ry0, ry1);
      __syncthreads();
    }
    // write back the core's points the chain wrote
    for (int b = 0; b < P->nbufs; b++) {
      const FBuf &B = P->B[b];
      double *dst = reinterpret_cast<double *>(B.dst);
      const double *srcs = sm + B.off;
      for (int k = 0; k < B.nwb; k++) {
        const int *wb = P->WB[B.wb0 + k];
        const int x0 = max(wb[0], c.cx0), x1 = min(wb[1], c.cx1);
        const int y0 = max(wb[2], c.cy0), y1 = min(wb[3], c.cy1);
        const int w = x1 - x0;
        if (w <= 0 || y1 <= y0) continue;
        double *d = dst + x0 + (long long)y0 * B.ay;
        const double *sv = srcs + (x0 - (c.cx0 - B.hx0)) + (y0 - (c.cy0 - B.hy0)) * B.pitch;
        const int dy = kThreads / w, dx = kThreads - dy * w;
        int yy = (int)threadIdx.x / w;
        int xx = (int)threadIdx.x - yy * w;
        for (; yy < y1 - y0;) {
          d[xx + (long long)yy * B.ay] = sv[xx + yy * B.pitch];
          xx += dx;
          yy += dy;
          if (xx >= w) {
            xx -= w;
            yy++;
          }
        }
      }
    }
    __syncthreads();
  }
  if (nred == 0) return;
  // reductions: per block, then across blocks by the last block to finish
  const int nblocks = gridDim.x;
  for (int r = 0; r < nred; r++) {
    double v = block_reduce<double>(racc[r], P->red[r].acc, red_smem);
    if (threadIdx.x == 0)
      reinterpret_cast<double *>(P->red_scratch)[((size_t)r * nblocks + blockIdx.x) * OPSB_MAX_RED_DIM] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned int done = atomicAdd(P->red_counter, 1u);
    last = (done == (unsigned int)(nblocks - 1));
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int r = 0; r < nred; r++) {
    const int acc = P->red[r].acc;
    double v = red_identity<double>(acc);
    const double *part = reinterpret_cast<const double *>(P->red_scratch) + (size_t)r * nblocks * OPSB_MAX_RED_DIM;
    for (int b = threadIdx.x; b < nblocks; b += kThreads) v = red_combine(acc, v, part[(size_t)b * OPSB_MAX_RED_DIM]);
    v = block_reduce<double>(v, acc, red_smem);
    if (threadIdx.x == 0) {
      double *slot = reinterpret_cast<double *>(P->red[r].slot);
      *slot = P->red[r].first ? v : red_combine(acc, *slot, v);
    }
  }
  if (threadIdx.x == 0) *P->red_counter = 0u;
}

// Registration of a group with the planner: kernel names in functor order.
struct GroupInfo {
  const char *name;
  int nkernels;
  const char *const *kernels;
  void (*launch)(const FPlan *, int grid, size_t smem_bytes, cudaStream_t);
  cudaError_t (*set_smem)(int bytes);
  int (*occupancy)(int smem_bytes);
};
void register_group(const GroupInfo &g);

template <class G>
void launch_group(const FPlan *p, int grid, size_t smem, cudaStream_t s) {
  fused_chain_kernel<G><<<grid, kThreads, smem, s>>>(p);
}
template <class G>
cudaError_t group_set_smem(int bytes) {
  return cudaFuncSetAttribute(fused_chain_kernel<G>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}
template <class G>
int group_occupancy(int smem) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fused_chain_kernel<G>, kThreads, smem) != cudaSuccess) return 0;
  return n;
}

template <int MinBlocks, class... K>
struct GroupRegistrar {
  GroupRegistrar(const char *name) {
    static const char *const names[] = {K::kname...};
    using G = Group<MinBlocks, K...>;
    GroupInfo g;
    g.name = name;
    g.nkernels = sizeof...(K);
    g.kernels = names;
    g.launch = &launch_group<G>;
    g.set_smem = &group_set_smem<G>;
    g.occupancy = &group_occupancy<G>;
    register_group(g);
  }
};

}  // namespace fuse
}  // namespace opsb
