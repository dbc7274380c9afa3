// Loop-chain fusion: one kernel runs a run of queued 2D loops tile by tile.
//
// The reference's lazy execution (ops/c/src/core/ops_lazy.cpp) queues loops
// until a sync point and, with OPS_TILING, builds a tile plan over them: a
// backward sweep over the queued loops' read/write ranges and stencils
// (ops_lazy.cpp:687-1114) gives every loop the extra iterations a tile needs
// so that later loops can read its results (halo depths, :1129-1173), and
// the plan is cached by the hash sequence of the queue (:1264-1283). On a CPU
// the tiles are sized for the last-level cache; on the GPU the reference
// runs one tile (:166), i.e. no fusion.
//
// Here the same analysis targets shared memory. A chain of loops runs in one
// persistent kernel over 2D tiles of TX x TY points ("the core"): each loop
// is applied to its core grown by its halo depths (recomputing the points a
// neighbouring tile also computes), and each dat is bound by what the chain
// does with it:
//   RO   never written in the chain: read from HBM through the read-only path;
//   RW   written, never read after a write in the chain, and no tile can read
//        a point another tile writes: read from HBM with coherent loads,
//        written to HBM only at the points of the tile's core;
//   TILE read after a write in the chain: a shared-memory tile covering the
//        core and every halo the chain reads it at. Staged from HBM first
//        when the chain reads values it had before the chain; written back
//        (the core's points the chain writes) at the end of the tile. When a
//        tile could read, before the chain writes it, a point that another
//        tile writes (a read at an offset, or by a loop with halo depths),
//        the dat is renamed: the chain stages from its current storage and
//        writes every point of its allocation back to a shadow allocation,
//        which becomes the dat's storage after the chain.
// Every per-point result equals the unfused loops' (each loop keeps its
// arithmetic, ranges and order); min/max reductions are order-independent,
// sum reductions end a chain.
#pragma once
#include <cuda_runtime.h>

namespace opsb {
namespace fuse {

constexpr int kMaxLoops = 96;    // loops in one chain (compute and boundary copies)
constexpr int kMaxArgs = 640;    // loop arguments over a chain
constexpr int kMaxBufs = 24;     // shared-memory tiles
constexpr int kMaxRed = 8;       // reduction arguments over a chain
constexpr int kMaxBoxes = 96;    // write-back boxes over all tiles
constexpr int kThreads = 256;
constexpr int kScratch = 16 + 24 + 16;  // per-thread masked-write cells (see TileCtx::scratch)
// Guard cells (zeros) around the shared-memory tiles, so that a kernel
// reading outside its declared stencil reads a wrong value (which the parity
// tests see) instead of leaving the shared-memory window.
constexpr int kGuard = 1024;

enum Mode : int { M_RO = 0, M_RW = 1, M_TILE = 2, M_GBL = 3, M_IDX = 4, M_RED = 5 };

struct FArg {
  char *ptr;   // RO/RW: logical origin of the dat's storage; GBL: device copy
  int sx, sy;  // point strides in elements (0 along a dimension the stencil does not walk)
  int ay;      // row pitch in elements
  int mode;
  int buf;     // TILE: shared-memory tile
  int red;     // RED: chain reduction slot
  int masked;  // RW written by this loop: points outside the core write a scratch cell
  int slot;    // that scratch cell: the argument's index in its loop (arguments must not alias)
};

struct FLoop {
  int kid;                 // functor index in the group; -1: boundary copy loop
  int x0, x1, y0, y1;      // iteration range
  int ex0, ex1, ey0, ey1;  // halo depths: the loop runs on [cx0-ex0, cx1+ex1) x [cy0-ey0, cy1+ey1)
  int arg0, nargs;         // this loop's arguments: A[arg0 .. arg0+nargs)
  // boundary copy loop: f(x,y) = (neg ? -1 : 1) * f(x+ox, y+oy) for the listed arguments
  int cp_n, cp_ox, cp_oy, cp_neg;
  int cp_arg[8];
};

struct FBuf {
  int hx0, hx1, hy0, hy1;  // halo around the core held by the tile
  int off;                 // offset in doubles in dynamic shared memory
  int pitch;               // TX + hx0 + hx1
  char *src;               // staging source (logical origin), nullptr: not staged
  char *dst;               // write-back destination (logical origin)
  int ay;                  // row pitch of src and dst (elements)
  int ax0, ax1, ay0, ay1;  // allocation box of the dat (logical, half-open)
  int wb0, nwb;            // write-back boxes WB[wb0 .. wb0+nwb)
};

struct FRed {
  char *slot;  // reduction handle's device slot
  int acc;     // ACC_MIN / ACC_MAX
  int first;   // 1: the handle restarts from the identity in this chain
};

struct FPlan {
  int TX, TY;
  int gx0, gy0, ntx, nty;  // tile grid: origin and tile counts
  int nloops, nbufs, nred;
  int smem_doubles;        // dynamic shared memory (guards included)
  char *red_scratch;
  unsigned int *red_counter;
  FRed red[kMaxRed];
  FLoop L[kMaxLoops];
  FBuf B[kMaxBufs];
  int WB[kMaxBoxes][4];    // x0, x1, y0, y1
  FArg A[kMaxArgs];
};

}  // namespace fuse
}  // namespace opsb
