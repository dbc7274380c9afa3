// Loop-chain fusion, host side: which runs of a flushed queue become one
// fused kernel, the analysis that makes it legal, the tile plan, and the
// choice of tile shape (see fusion.h for the binding rules).
//
// Analysis of a candidate chain (the counterpart of ops_construct_tile_plan,
// ops/c/src/core/ops_lazy.cpp:380, and its dependency sweep, :687-1114):
//  1. every dat access of every loop: read and/or written, the bounding box
//     of the stencil (a boundary copy loop reads its mirror offset and
//     writes its point, for the fields its flags select);
//  2. halo depths, backwards: a loop that reads dat f at stencil box S over
//     its region (core + depths) needs every earlier loop writing f (whose
//     range meets the read) to run on that region grown by S;
//  3. per dat, the binding: RO / RW / TILE, staged or not, renamed or not
//     (box arithmetic over the loops' ranges decides which reads see values
//     from before the chain and whether such a read can meet a point that
//     the chain writes);
//  4. the compulsory bytes of the fused chain (each dat's points read once
//     from HBM and written once), against the sum of the loops' own.
// The tile shape is tuned per chain structure: the first executions of a
// chain try each candidate shape (all give identical results) timed with
// CUDA events, the fastest is kept and written to a cache file
// (OPS_B200_TUNE_CACHE, default ~/.cache/ops_b200/fusion_tiles.txt), which
// later runs read instead of tuning again.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <set>
#include <sstream>
#include <sys/stat.h>

#include "fused_exec.cuh"
#include "runtime.h"

namespace opsb {
namespace fuse {

std::vector<GroupInfo> &groups() {
  static std::vector<GroupInfo> g;
  return g;
}
void register_group(const GroupInfo &g) { groups().push_back(g); }

}  // namespace fuse

namespace {
using namespace fuse;

struct B2 {
  int x0, x1, y0, y1;  // half-open
  bool empty() const { return x0 >= x1 || y0 >= y1; }
  long long area() const { return empty() ? 0 : (long long)(x1 - x0) * (y1 - y0); }
};
B2 inter(const B2 &a, const B2 &b) {
  return {std::max(a.x0, b.x0), std::min(a.x1, b.x1), std::max(a.y0, b.y0), std::min(a.y1, b.y1)};
}
B2 hull(const B2 &a, const B2 &b) {
  if (a.empty()) return b;
  if (b.empty()) return a;
  return {std::min(a.x0, b.x0), std::max(a.x1, b.x1), std::min(a.y0, b.y0), std::max(a.y1, b.y1)};
}
bool inside(int x, int y, const B2 &b) { return x >= b.x0 && x < b.x1 && y >= b.y0 && y < b.y1; }

// Is there a point of R that lies in some box of `in` (every point of R
// when `in_all` is set) and in no box of `out`? Exact, by coordinate
// compression over the boxes' edges.
bool exists_point(const B2 &R, const std::vector<B2> &in, bool in_all, const std::vector<B2> &out) {
  if (R.empty()) return false;
  std::vector<int> xs{R.x0, R.x1}, ys{R.y0, R.y1};
  auto add = [&](const B2 &b) {
    for (int v : {b.x0, b.x1})
      if (v > R.x0 && v < R.x1) xs.push_back(v);
    for (int v : {b.y0, b.y1})
      if (v > R.y0 && v < R.y1) ys.push_back(v);
  };
  for (const B2 &b : in) add(b);
  for (const B2 &b : out) add(b);
  std::sort(xs.begin(), xs.end());
  xs.erase(std::unique(xs.begin(), xs.end()), xs.end());
  std::sort(ys.begin(), ys.end());
  ys.erase(std::unique(ys.begin(), ys.end()), ys.end());
  for (size_t a = 0; a + 1 < xs.size(); a++)
    for (size_t b = 0; b + 1 < ys.size(); b++) {
      const int x = xs[a], y = ys[b];  // a representative point of this cell
      bool ok = in_all;
      if (!in_all)
        for (const B2 &q : in) ok = ok || inside(x, y, q);
      if (!ok) continue;
      bool excluded = false;
      for (const B2 &q : out) excluded = excluded || inside(x, y, q);
      if (!excluded) return true;
    }
  return false;
}

constexpr int kMaxDepth = 3;              // deepest halo a chain may need (recompute grows with it)
constexpr int kSmemBudget = 220 * 1024;   // dynamic shared memory per CTA
struct Shape { int tx, ty; };
const Shape kShapes[] = {{64, 8}, {128, 8}, {64, 16}, {128, 16}, {32, 16}};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);
// Tuning candidates: a tile shape, with the read-only dats read from HBM in
// the loops (even index) or staged into shared memory with the rest at the
// start of each tile (odd index); the last candidate runs the chain's loops
// one by one, unfused.
constexpr int kNumCands = 2 * kNumShapes;
constexpr int kUnfused = kNumCands;
inline const Shape &cand_shape(int c) { return kShapes[c / 2]; }
inline bool cand_stage_ro(int c) { return (c & 1) != 0; }

struct DatAccess {
  int loop, arg, dat;
  bool rd, wr, edge;
  B2 st;  // stencil box (offsets, half-open: [min, max+1))
};

struct FieldInfo {
  int dat = -1;
  int mode = M_RO;
  bool staged = false, renamed = false;
  bool stageable = false;  // RO, a 2D double dat: may be staged into a read-only tile
  int hx0 = 0, hx1 = 0, hy0 = 0, hy1 = 0;
  std::vector<B2> writes;  // ranges of the loops writing it
  B2 alloc{0, 0, 0, 0};
  B2 pre{0, 0, 0, 0};      // hull of the points read with their value from before the chain
};

struct LoopInfoF {
  int kid = -1;
  bool copy = false;
  int ex0 = 0, ex1 = 0, ey0 = 0, ey1 = 0;
  B2 range;
  std::vector<int> cp_args;  // copy loop: argument indices whose flag is set
};

bool trace_on() {
  static const bool t = getenv("OPS_B200_FUSION_TRACE") != nullptr;
  return t;
}

// Rejections that a longer chain cannot undo: the greedy growth stops there.
bool final_rejection(const std::string &why) {
  return why == "halo depth above the limit" || why == "too many loops" || why == "too many arguments" ||
         why == "too many tiles" || why == "kernels of two fusion groups" || why == "too many reductions" ||
         why.rfind("an edge", 0) == 0;
}

}  // namespace

// Everything the planner decides for one chain, independent of the tile
// shape and of the dats' storage addresses.
struct ChainAnalysis {
  size_t first = 0, n = 0;
  int group = -1;
  std::vector<LoopInfoF> loops;
  std::vector<DatAccess> acc;
  std::map<int, FieldInfo> fields;  // by dat index
  int nred = 0;
  double fused_bytes = 0, loop_bytes = 0;
  uint64_t key = 0;  // structure hash
  std::string why;   // reason for rejection
};

class FusionPlanner {
 public:
  explicit FusionPlanner(Runtime &r) : rt(r) {}

  static const std::pair<int, int> *find_kernel(const std::string &name) {
    static std::map<std::string, std::pair<int, int>> m;
    static size_t built = 0;
    if (built != groups().size()) {
      m.clear();
      for (size_t g = 0; g < groups().size(); g++)
        for (int k = 0; k < groups()[g].nkernels; k++) m[groups()[g].kernels[k]] = {(int)g, k};
      built = groups().size();
    }
    auto it = m.find(name);
    return it == m.end() ? nullptr : &it->second;
  }

  // Can loop d be part of a chain at all (independent of its neighbours)?
  bool eligible(const Desc &d, int *group) const {
    if (d.loop->internal || d.dim != 2 || d.loop->ndim > 2) return false;
    const CopyLoopSpec *sp = find_copy_loop(d.loop);
    if (sp) {
      if (sp->off[2] != 0 || sp->nfields > 8) return false;
      *group = -1;
    } else {
      const auto *k = find_kernel(d.loop->kernel);
      if (!k) return false;
      *group = k->first;
    }
    for (const Arg &a : d.args) {
      switch (a.kind) {
        case ARG_DAT: {
          const Dat &dt = *rt.dats_[a.dat];
          const Stencil &st = rt.stencils_[a.stencil];
          if (st.type != 0 || dt.dim != 1) return false;
          if (a.acc != ACC_READ && (dt.elem_size != 8 || !st.stride[0] || !st.stride[1])) return false;
          if (a.acc == ACC_INC || a.acc == ACC_MIN || a.acc == ACC_MAX) return false;
          break;
        }
        case ARG_GBL:
          if (a.acc != ACC_READ) return false;
          break;
        case ARG_REDUCE:
          if ((a.acc != ACC_MIN && a.acc != ACC_MAX) || a.dim != 1 || a.elem != 8) return false;
          break;
        case ARG_IDX:
          break;
        default:
          return false;
      }
    }
    return true;
  }

  static B2 stencil_box(const Stencil &st, bool *edge) {
    int mn[2] = {0, 0}, mx[2] = {0, 0};
    *edge = false;
    for (int k = 0; k < 2; k++) {
      if (!st.stride[k]) {
        *edge = true;
        continue;
      }
      for (int p = 0; p < st.points; p++) {
        const int o = st.offs[(size_t)p * st.dims + k];
        if (p == 0 || o < mn[k]) mn[k] = o;
        if (p == 0 || o > mx[k]) mx[k] = o;
      }
    }
    return {mn[0], mx[0] + 1, mn[1], mx[1] + 1};
  }

  B2 alloc_box(const Dat &d) const {
    return {d.lo[0], d.hi[0], d.lo[1], d.hi[1]};
  }

  // Steps 1-4 of the analysis for q[first, first+n).
  bool analyse(const std::vector<Desc> &q, size_t first, size_t n, ChainAnalysis &A) const {
    A = ChainAnalysis();
    A.first = first;
    A.n = n;
    if (n > (size_t)kMaxLoops) return reject(A, "too many loops");
    uint64_t h = 0xCBF29CE484222325ULL;
    auto mix = [&h](uint64_t v) { h = (h ^ v) * 0x100000001B3ULL; };
    int ncompute = 0, nargs = 0;
    for (size_t l = 0; l < n; l++) {
      const Desc &d = q[first + l];
      LoopInfoF li;
      li.range = {d.range[0], d.range[1], d.range[2], d.range[3]};
      int g = -1;
      if (!eligible(d, &g)) return reject(A, "ineligible loop " + d.loop->kernel);
      const CopyLoopSpec *sp = find_copy_loop(d.loop);
      mix(std::hash<std::string>()(d.loop->kernel));
      for (int k = 0; k < 4; k++) mix((uint64_t)(uint32_t)d.range[k]);
      if (sp) {
        li.copy = true;
        const int *flags =
            sp->flags_arg >= 0 ? reinterpret_cast<const int *>(d.args[sp->flags_arg].gbl.data()) : nullptr;
        const int nflags = sp->flags_arg >= 0 ? (int)(d.args[sp->flags_arg].gbl.size() / sizeof(int)) : 0;
        for (int f = 0; f < sp->nfields; f++) {
          if (flags && (sp->flag[f] >= nflags || flags[sp->flag[f]] != 1)) continue;
          const Arg &a = d.args[sp->arg[f]];
          li.cp_args.push_back(sp->arg[f]);
          mix((uint64_t)a.dat * 31 + f);
          A.acc.push_back({(int)l, sp->arg[f], a.dat, true, false, false,
                           {sp->off[0], sp->off[0] + 1, sp->off[1], sp->off[1] + 1}});
          A.acc.push_back({(int)l, sp->arg[f], a.dat, false, true, false, {0, 1, 0, 1}});
        }
      } else {
        ncompute++;
        if (A.group < 0) A.group = g;
        if (g != A.group) return reject(A, "kernels of two fusion groups");
        li.kid = find_kernel(d.loop->kernel)->second;
        for (size_t i = 0; i < d.args.size(); i++) {
          const Arg &a = d.args[i];
          mix(((uint64_t)a.kind << 40) ^ ((uint64_t)a.acc << 32) ^ (uint64_t)(uint32_t)a.stencil);
          if (a.kind == ARG_REDUCE) A.nred++;
          if (a.kind != ARG_DAT) continue;
          mix((uint64_t)a.dat);
          bool edge = false;
          B2 st = stencil_box(rt.stencils_[a.stencil], &edge);
          const bool rd = a.acc == ACC_READ || a.acc == ACC_RW;
          const bool wr = a.acc == ACC_WRITE || a.acc == ACC_RW;
          A.acc.push_back({(int)l, (int)i, a.dat, rd, wr, edge, st});
        }
      }
      nargs += (int)d.args.size();
      A.loops.push_back(li);
    }
    A.key = h;
    if (ncompute < 2) return reject(A, "fewer than two compute loops");
    if (A.group < 0) return reject(A, "no compute loop");
    if (nargs > kMaxArgs) return reject(A, "too many arguments");
    if (A.nred > kMaxRed) return reject(A, "too many reductions");

    // 2. halo depths, backwards
    for (int i = (int)n - 1; i >= 0; i--) {
      LoopInfoF &Li = A.loops[i];
      for (const DatAccess &r : A.acc) {
        if (r.loop != i || !r.rd) continue;
        const B2 rbox{Li.range.x0 + r.st.x0, Li.range.x1 + r.st.x1 - 1, Li.range.y0 + r.st.y0,
                      Li.range.y1 + r.st.y1 - 1};
        for (const DatAccess &w : A.acc) {
          if (w.loop >= i || !w.wr || w.dat != r.dat) continue;
          LoopInfoF &Lj = A.loops[w.loop];
          if (inter(Lj.range, rbox).empty()) continue;
          Lj.ex0 = std::max(Lj.ex0, Li.ex0 - r.st.x0);
          Lj.ex1 = std::max(Lj.ex1, Li.ex1 + r.st.x1 - 1);
          Lj.ey0 = std::max(Lj.ey0, Li.ey0 - r.st.y0);
          Lj.ey1 = std::max(Lj.ey1, Li.ey1 + r.st.y1 - 1);
        }
      }
    }
    for (const LoopInfoF &L : A.loops)
      if (std::max({L.ex0, L.ex1, L.ey0, L.ey1}) > kMaxDepth) return reject(A, "halo depth above the limit");

    // 3. bindings
    for (const DatAccess &a : A.acc) {
      FieldInfo &f = A.fields[a.dat];
      f.dat = a.dat;
      f.alloc = alloc_box(*rt.dats_[a.dat]);
      if (a.wr) f.writes.push_back(A.loops[a.loop].range);
    }
    for (auto &kv : A.fields) {
      FieldInfo &f = kv.second;
      bool raw = false, pre = false, hazard = false, edge = false, self_rw = false;
      for (const DatAccess &a : A.acc) {
        if (a.dat != f.dat) continue;
        const LoopInfoF &L = A.loops[a.loop];
        edge = edge || a.edge;
        if (!a.rd) continue;
        const B2 box{L.range.x0 + a.st.x0, L.range.x1 + a.st.x1 - 1, L.range.y0 + a.st.y0, L.range.y1 + a.st.y1 - 1};
        std::vector<B2> prior;
        for (const DatAccess &w : A.acc)
          if (w.dat == f.dat && w.wr && w.loop < a.loop) prior.push_back(A.loops[w.loop].range);
        if (exists_point(box, prior, false, {})) raw = true;
        const bool grown = L.ex0 || L.ex1 || L.ey0 || L.ey1;
        if (exists_point(box, {}, true, prior)) {
          pre = true;
          f.pre = hull(f.pre, inter(box, f.alloc));
          const bool offset = !(a.st.x0 == 0 && a.st.x1 == 1 && a.st.y0 == 0 && a.st.y1 == 1);
          if ((offset || grown) && exists_point(box, f.writes, false, prior)) hazard = true;
        }
        // a kernel (not a copy loop) that reads and writes f and runs on
        // points outside the core: its writes there cannot be dropped
        if (!L.copy && grown)
          for (const DatAccess &w : A.acc)
            if (w.loop == a.loop && w.dat == f.dat && w.wr) self_rw = true;
      }
      if (f.writes.empty()) {
        f.mode = M_RO;
        f.stageable = !edge && rt.dats_[f.dat]->elem_size == 8;
      } else if (!raw && !hazard && !self_rw) {
        f.mode = M_RW;
      } else {
        if (edge || rt.dats_[f.dat]->elem_size != 8) return reject(A, "an edge or non-double dat needs a tile");
        f.mode = M_TILE;
        f.renamed = hazard;
        f.staged = pre || hazard;
      }
    }
    // tile halos: every access's reach around the core
    for (const DatAccess &a : A.acc) {
      FieldInfo &f = A.fields[a.dat];
      if (f.mode != M_TILE && !f.stageable) continue;
      const LoopInfoF &L = A.loops[a.loop];
      f.hx0 = std::max(f.hx0, L.ex0 - a.st.x0);
      f.hx1 = std::max(f.hx1, L.ex1 + a.st.x1 - 1);
      f.hy0 = std::max(f.hy0, L.ey0 - a.st.y0);
      f.hy1 = std::max(f.hy1, L.ey1 + a.st.y1 - 1);
    }
    int nbufs = 0;
    for (auto &kv : A.fields) nbufs += kv.second.mode == M_TILE || kv.second.stageable;
    if (nbufs > kMaxBufs) return reject(A, "too many tiles");

    // 4. bytes: the fused chain's compulsory traffic against the loops' own
    for (auto &kv : A.fields) {
      const FieldInfo &f = kv.second;
      double rd = 0, wr = 0;
      B2 wh{0, 0, 0, 0};
      for (const B2 &w : f.writes) wh = hull(wh, inter(w, f.alloc));
      if (f.mode == M_TILE && f.renamed) {
        rd = wr = (double)f.alloc.area();
      } else {
        rd = (double)f.pre.area();
        wr = (double)wh.area();
      }
      A.fused_bytes += 8.0 * (rd + wr);
    }
    for (size_t l = 0; l < n; l++) A.loop_bytes += rt.alg_bytes(q[first + l]);
    if (!(A.fused_bytes < 0.95 * A.loop_bytes)) return reject(A, "no traffic saved");
    return true;
  }

  // Shared memory of a chain at a tile shape, in doubles (guards included).
  static int smem_doubles(const ChainAnalysis &A, int TX, int TY, bool stage_ro) {
    long long s = 2 * kGuard;
    for (const auto &kv : A.fields) {
      const FieldInfo &f = kv.second;
      if (f.mode != M_TILE && !(stage_ro && f.stageable)) continue;
      s += (long long)(TX + f.hx0 + f.hx1) * (TY + f.hy0 + f.hy1);
    }
    return (int)std::min<long long>(s, 1LL << 30);
  }

  // The device plan at a tile shape; renames are applied to the runtime's
  // dats (the chain writes the renamed dats into their shadow storage).
  void build(const std::vector<Desc> &q, const ChainAnalysis &A, int TX, int TY, bool stage_ro, FPlan &P,
             std::vector<int> &renamed) {
    memset(&P, 0, sizeof(P));
    P.TX = TX;
    P.TY = TY;
    B2 grid{0, 0, 0, 0};
    for (const LoopInfoF &L : A.loops) grid = hull(grid, L.range);
    for (const auto &kv : A.fields)
      if (kv.second.mode == M_TILE && kv.second.renamed) grid = hull(grid, kv.second.alloc);
    P.gx0 = grid.x0;
    P.gy0 = grid.y0;
    P.ntx = (grid.x1 - grid.x0 + TX - 1) / TX;
    P.nty = (grid.y1 - grid.y0 + TY - 1) / TY;
    // tiles
    std::map<int, int> buf_of;
    int off = 0, nwb = 0;
    for (const auto &kv : A.fields) {
      const FieldInfo &f = kv.second;
      const bool ro_tile = stage_ro && f.stageable;
      if (f.mode != M_TILE && !ro_tile) continue;
      const int b = P.nbufs++;
      buf_of[f.dat] = b;
      FBuf &B = P.B[b];
      Dat &d = *rt.dats_[f.dat];
      B.hx0 = f.hx0; B.hx1 = f.hx1; B.hy0 = f.hy0; B.hy1 = f.hy1;
      B.pitch = TX + f.hx0 + f.hx1;
      B.off = off;
      off += B.pitch * (TY + f.hy0 + f.hy1);
      B.ay = (int)d.pitch;
      B.ax0 = f.alloc.x0; B.ax1 = f.alloc.x1; B.ay0 = f.alloc.y0; B.ay1 = f.alloc.y1;
      char *cur = d.origin_ptr();
      B.src = (f.staged || ro_tile) ? cur : nullptr;
      if (ro_tile) {  // read-only: staged, never written back
        B.dst = nullptr;
        B.wb0 = nwb;
        B.nwb = 0;
      } else if (f.renamed) {
        char *&sh = rt.shadow_[f.dat];
        if (!sh) sh = rt.alloc_dat_storage(d.bytes);
        std::swap(d.data_d, sh);  // the dat now lives in the former shadow
        d.host.clear();
        renamed.push_back(f.dat);
        B.dst = d.origin_ptr();
        B.wb0 = nwb;
        B.nwb = 1;
        P.WB[nwb][0] = f.alloc.x0; P.WB[nwb][1] = f.alloc.x1; P.WB[nwb][2] = f.alloc.y0; P.WB[nwb][3] = f.alloc.y1;
        nwb++;
      } else {
        B.dst = cur;
        B.wb0 = nwb;
        for (const B2 &w : f.writes) {
          const B2 c = inter(w, f.alloc);
          if (c.empty()) continue;
          if (nwb >= kMaxBoxes) throw Error(E_UNSUPPORTED, "fusion: too many write-back boxes");
          P.WB[nwb][0] = c.x0; P.WB[nwb][1] = c.x1; P.WB[nwb][2] = c.y0; P.WB[nwb][3] = c.y1;
          nwb++;
        }
        B.nwb = nwb - B.wb0;
      }
    }
    P.smem_doubles = off + 2 * kGuard;
    // loops and arguments
    int na = 0;
    for (size_t l = 0; l < A.n; l++) {
      const Desc &d = q[A.first + l];
      const LoopInfoF &Li = A.loops[l];
      FLoop &L = P.L[P.nloops++];
      L.kid = Li.copy ? -1 : Li.kid;
      L.x0 = Li.range.x0; L.x1 = Li.range.x1; L.y0 = Li.range.y0; L.y1 = Li.range.y1;
      L.ex0 = Li.ex0; L.ex1 = Li.ex1; L.ey0 = Li.ey0; L.ey1 = Li.ey1;
      L.arg0 = na;
      L.nargs = (int)d.args.size();
      if (Li.copy) {
        const CopyLoopSpec *sp = find_copy_loop(d.loop);
        L.cp_n = (int)Li.cp_args.size();
        for (int f = 0; f < L.cp_n; f++) L.cp_arg[f] = Li.cp_args[f];
        L.cp_ox = sp->off[0];
        L.cp_oy = sp->off[1];
        L.cp_neg = sp->neg;
      }
      for (size_t i = 0; i < d.args.size(); i++) {
        const Arg &a = d.args[i];
        FArg &F = P.A[na++];
        switch (a.kind) {
          case ARG_DAT: {
            const Dat &dt = *rt.dats_[a.dat];
            const Stencil &st = rt.stencils_[a.stencil];
            F.ptr = dt.origin_ptr();
            F.sx = st.stride[0] ? 1 : 0;
            F.sy = st.stride[1] ? (int)dt.pitch : 0;
            F.ay = (int)dt.pitch;
            auto fit = A.fields.find(a.dat);
            if (fit == A.fields.end()) {  // a copy loop's field whose flag is off: never accessed
              F.mode = M_RO;
              break;
            }
            const FieldInfo &f = fit->second;
            F.mode = f.mode;
            if (buf_of.count(a.dat)) {
              F.mode = M_TILE;
              F.buf = buf_of.at(a.dat);
            }
            F.masked = f.mode == M_RW && (a.acc == ACC_WRITE || a.acc == ACC_RW);
            F.slot = (int)i;
            break;
          }
          case ARG_GBL:
            F.mode = M_GBL;
            F.ptr = rt.gbl_dev_ + d.gbl_off[i];
            break;
          case ARG_IDX:
            F.mode = M_IDX;
            break;
          case ARG_REDUCE: {
            F.mode = M_RED;
            F.red = P.nred;
            FRed &R = P.red[P.nred++];
            R.slot = rt.reductions_[a.red].slot_d;
            R.acc = a.acc;
            R.first = d.red_first[i];
            break;
          }
        }
      }
    }
    P.red_scratch = rt.red_scratch_;
    validate(A, P, buf_of);
  }

  // Every shared-memory access the plan allows stays inside its tile: each
  // access's reach (the loop's halo depths grown by the stencil box) within
  // the tile's halo, write-back boxes within the allocation, the tiles within
  // the shared memory. Checked on the host for every plan built.
  static void validate(const ChainAnalysis &A, const FPlan &P, const std::map<int, int> &buf_of) {
    for (const DatAccess &a : A.acc) {
      if (!buf_of.count(a.dat)) continue;
      const FLoop &L = P.L[a.loop];
      const FArg &F = P.A[L.arg0 + a.arg];
      if (F.mode != M_TILE || F.buf < 0 || F.buf >= P.nbufs) throw Error(E_STATE, "fusion plan: tile binding");
      const FBuf &B = P.B[F.buf];
      if (L.ex0 - a.st.x0 > B.hx0 || L.ex1 + a.st.x1 - 1 > B.hx1 || L.ey0 - a.st.y0 > B.hy0 ||
          L.ey1 + a.st.y1 - 1 > B.hy1)
        throw Error(E_STATE, "fusion plan: an access reaches outside its shared-memory tile");
    }
    long long end = 0;
    for (int b = 0; b < P.nbufs; b++) {
      const FBuf &B = P.B[b];
      if (B.pitch != P.TX + B.hx0 + B.hx1 || B.off != end) throw Error(E_STATE, "fusion plan: tile layout");
      end += (long long)B.pitch * (P.TY + B.hy0 + B.hy1);
      for (int k = 0; k < B.nwb; k++) {
        const int *w = P.WB[B.wb0 + k];
        if (w[0] < B.ax0 || w[1] > B.ax1 || w[2] < B.ay0 || w[3] > B.ay1)
          throw Error(E_STATE, "fusion plan: write-back outside the allocation");
      }
    }
    if (end + 2 * kGuard != P.smem_doubles || P.smem_doubles * 8 > kSmemBudget)
      throw Error(E_STATE, "fusion plan: shared memory size");
  }

  static void trace(const std::vector<Desc> &q, const ChainAnalysis &A, const Runtime &r) {
    fprintf(stderr, "fused chain [%zu, %zu): %zu loops\n", A.first, A.first + A.n, A.n);
    for (size_t l = 0; l < A.n; l++) {
      const LoopInfoF &L = A.loops[l];
      fprintf(stderr, "  %-40s halo x-%d x+%d y-%d y+%d\n", q[A.first + l].loop->kernel.c_str(), L.ex0, L.ex1, L.ey0,
              L.ey1);
    }
    for (const auto &kv : A.fields) {
      const FieldInfo &f = kv.second;
      static const char *mn[] = {"RO", "RW", "TILE"};
      fprintf(stderr, "  dat %-14s %s%s%s halo %d %d %d %d\n", r.dats_[f.dat]->name.c_str(), mn[f.mode],
              f.staged ? " staged" : "", f.renamed ? " renamed" : "", f.hx0, f.hx1, f.hy0, f.hy1);
    }
    fprintf(stderr, "  bytes fused %.3e, as loops %.3e\n", A.fused_bytes, A.loop_bytes);
  }

  Runtime &rt;

 private:
  static bool reject(ChainAnalysis &A, const std::string &why) {
    A.why = why;
    return false;
  }
};

// ---------------------------------------------------------------------------
// Tile-shape tuning state and its cache file.
// ---------------------------------------------------------------------------
struct FusionState {
  struct Tune {
    int chosen = -1;
    int next = 0;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;  // shape, events
    std::vector<double> ms = std::vector<double>(kNumCands + 1, 1e30);
  };
  std::map<uint64_t, Tune> tune;
  bool loaded = false;
  std::string path;
  std::vector<cudaEvent_t> free_events;
  // device copies of plans, by content hash
  std::map<uint64_t, std::pair<FPlan *, std::unique_ptr<FPlan>>> plans;
  // chain boundaries of a queue structure (first, n), by the queue's hash
  std::map<uint64_t, std::vector<std::pair<size_t, size_t>>> bounds;
  std::map<std::pair<int, int>, int> occupancy;  // (group, smem bytes) -> CTAs per SM
  std::set<int> smem_set;

  void drop_plans() {
    for (auto &kv : plans)
      if (kv.second.first) cudaFree(kv.second.first);
    plans.clear();
    bounds.clear();
  }

  ~FusionState() {
    for (auto &kv : plans)
      if (kv.second.first) cudaFree(kv.second.first);
    for (auto &kv : tune)
      for (auto &p : kv.second.pending) {
        cudaEventDestroy(p.second.first);
        cudaEventDestroy(p.second.second);
      }
    for (cudaEvent_t e : free_events) cudaEventDestroy(e);
  }

  cudaEvent_t event() {
    if (free_events.empty()) {
      cudaEvent_t e;
      OPSB_CUDA(cudaEventCreate(&e));
      return e;
    }
    cudaEvent_t e = free_events.back();
    free_events.pop_back();
    return e;
  }

  void load() {
    if (loaded) return;
    loaded = true;
    const char *p = getenv("OPS_B200_TUNE_CACHE");
    if (p) {
      path = p;
    } else {
      const char *home = getenv("HOME");
      path = std::string(home ? home : "/tmp") + "/.cache/ops_b200/fusion_tiles.txt";
    }
    std::ifstream in(path);
    std::string line;
    while (std::getline(in, line)) {
      std::istringstream ls(line);
      std::string key;
      int tx = 0, ty = 0, ro = 0;
      if (!(ls >> key >> tx >> ty)) continue;
      if (!(ls >> ro)) ro = 0;
      if (tx == 0 && ty == 0) tune[std::stoull(key, nullptr, 16)].chosen = kUnfused;
      for (int s = 0; s < kNumShapes; s++)
        if (kShapes[s].tx == tx && kShapes[s].ty == ty) tune[std::stoull(key, nullptr, 16)].chosen = 2 * s + (ro ? 1 : 0);
    }
  }

  void save(uint64_t key, int s) {
    if (path.empty()) return;
    const size_t slash = path.rfind('/');
    if (slash != std::string::npos) {
      // create the directories (mkdir -p), ignoring failures: the cache is optional
      std::string dir = path.substr(0, slash);
      for (size_t k = 1; k <= dir.size(); k++)
        if (k == dir.size() || dir[k] == '/') mkdir(dir.substr(0, k).c_str(), 0755);
    }
    std::ofstream out(path, std::ios::app);
    if (out) {
      char buf[64];
      snprintf(buf, sizeof(buf), "%016llx %d %d %d\n", (unsigned long long)key, s == kUnfused ? 0 : cand_shape(s).tx,
               s == kUnfused ? 0 : cand_shape(s).ty, s == kUnfused ? 0 : (int)cand_stage_ro(s));
      out << buf;
    }
  }

  // Folds finished timings in; returns the shape to use (-1: none fits) and
  // whether this execution measures a candidate.
  int shape_for(uint64_t key, const std::vector<int> &fits, bool tuning_on, bool *tuning) {
    Tune &T = tune[key];
    *tuning = false;
    if (T.chosen >= 0 && std::find(fits.begin(), fits.end(), T.chosen) != fits.end()) return T.chosen;
    if (fits.empty()) return -1;
    if (!tuning_on) return fits[0];
    for (auto it = T.pending.begin(); it != T.pending.end();) {
      if (cudaEventQuery(it->second.second) != cudaSuccess) {
        ++it;
        continue;
      }
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, it->second.first, it->second.second) == cudaSuccess)
        T.ms[it->first] = std::min(T.ms[it->first], (double)ms);
      free_events.push_back(it->second.first);
      free_events.push_back(it->second.second);
      it = T.pending.erase(it);
    }
    bool all = true;
    for (int s : fits) all = all && T.ms[s] < 1e29;
    if (all && T.pending.empty()) {
      int best = fits[0];
      for (int s : fits)
        if (T.ms[s] < T.ms[best]) best = s;
      T.chosen = best;
      save(key, best);
      if (trace_on()) {
        fprintf(stderr, "tuned chain %016llx:", (unsigned long long)key);
        for (int s : fits)
          fprintf(stderr, " %s=%.4fms", s == kUnfused ? "unfused"
                                                      : (std::to_string(cand_shape(s).tx) + "x" +
                                                         std::to_string(cand_shape(s).ty) + (cand_stage_ro(s) ? "s" : ""))
                                                            .c_str(),
                  T.ms[s]);
        fprintf(stderr, " -> %s\n", best == kUnfused ? "unfused" : "fused");
      }
      return best;
    }
    *tuning = true;
    for (size_t k = 0; k < fits.size(); k++) {
      const int s = fits[(T.next + k) % fits.size()];
      if (T.ms[s] >= 1e29) {
        T.next = (int)((T.next + k + 1) % fits.size());
        return s;
      }
    }
    return fits[0];
  }
};

// ---------------------------------------------------------------------------
// Runtime hooks
// ---------------------------------------------------------------------------
FusionState &Runtime::fusion_state() {
  if (!fusion_state_) fusion_state_ = new FusionState();
  return *fusion_state_;
}
// An app call's end: its plans (which hold its dats' addresses) go; the
// tile-shape tuning state stays for the next calls of the same chains.
void Runtime::release_fusion_plans() {
  if (fusion_state_) fusion_state_->drop_plans();
}
void Runtime::set_tile_candidate(int c) {
  if (c < -1 || c >= kNumCands) throw Error(E_ARG, "tile_candidate must be -1 or 0.." + std::to_string(kNumCands - 1));
  tile_candidate_ = c;
}
void Runtime::release_fusion_state() {
  delete fusion_state_;
  fusion_state_ = nullptr;
}

// Chooses the fused chains of q and their tile shapes (no storage moves
// yet): `items` in queue order.
void Runtime::plan_fusion(const std::vector<Desc> &q, std::vector<FusedItem> &items) {
  items.clear();
  if (!fusion_on_ || !tiling_on_ || fuse::groups().empty()) return;
  FusionState &S = fusion_state();
  S.load();
  FusionPlanner fp(*this);
  // chain boundaries of this queue structure
  uint64_t qk = 0xCBF29CE484222325ULL;
  for (const Desc &d : q) {
    qk = (qk ^ (uint64_t)(uintptr_t)d.loop) * 0x100000001B3ULL;
    for (int k = 0; k < 4; k++) qk = (qk ^ (uint64_t)(uint32_t)d.range[k]) * 0x100000001B3ULL;
    for (const Arg &a : d.args) {
      qk = (qk ^ (((uint64_t)(uint32_t)a.dat << 32) ^ ((uint64_t)a.acc << 24) ^ (uint64_t)(uint32_t)a.stencil)) *
           0x100000001B3ULL;
      if (a.kind == ARG_GBL)
        for (char c : a.gbl) qk = (qk ^ (uint64_t)(unsigned char)c) * 0x100000001B3ULL;
    }
  }
  auto bit = S.bounds.find(qk);
  if (bit == S.bounds.end()) {
    std::vector<std::pair<size_t, size_t>> b;
    size_t i = 0;
    while (i < q.size()) {
      int g;
      if (!fp.eligible(q[i], &g)) {
        i++;
        continue;
      }
      // the chain from i that saves the most HBM traffic
      size_t best = 0;
      double best_saved = 0.0;
      ChainAnalysis A;
      for (size_t j = i + 1; j <= q.size(); j++) {
        int gj;
        if (!fp.eligible(q[j - 1], &gj)) break;
        if (fp.analyse(q, i, j - i, A)) {
          const double saved = A.loop_bytes - A.fused_bytes;
          if (saved > best_saved) {
            best = j - i;
            best_saved = saved;
          }
        } else {
          if (trace_on() && A.why != "fewer than two compute loops")
            fprintf(stderr, "  chain [%zu, %zu) rejected: %s\n", i, j, A.why.c_str());
          if (final_rejection(A.why)) break;
        }
      }
      if (best > 0) {
        b.push_back({i, best});
        i += best;
      } else {
        i++;
      }
    }
    bit = S.bounds.emplace(qk, std::move(b)).first;
  }
  const bool tuning_on = !(getenv("OPS_B200_TUNE") && atoi(getenv("OPS_B200_TUNE")) == 0);
  const bool trace = trace_on();
  for (const auto &fb : bit->second) {
    auto A = std::make_shared<ChainAnalysis>();
    if (!fp.analyse(q, fb.first, fb.second, *A)) continue;  // the structure was analysed before
    const fuse::GroupInfo &G = fuse::groups()[A->group];
    std::vector<int> fits;
    for (int s = 0; s < kNumCands; s++) {
      const int smem = FusionPlanner::smem_doubles(*A, cand_shape(s).tx, cand_shape(s).ty, cand_stage_ro(s)) * 8;
      if (smem > kSmemBudget) continue;
      auto ok = S.occupancy.find({A->group, smem});
      if (ok == S.occupancy.end()) {
        if (!S.smem_set.count(A->group)) {
          OPSB_CUDA(G.set_smem(kSmemBudget));
          S.smem_set.insert(A->group);
        }
        ok = S.occupancy.emplace(std::make_pair(A->group, smem), G.occupancy(smem)).first;
      }
      if (ok->second > 0) fits.push_back(s);
    }
    bool tuning = false;
    int s;
    if (tile_candidate_ >= 0) {  // one candidate for every chain it fits (tests, profiling): no tuning
      if (std::find(fits.begin(), fits.end(), tile_candidate_) == fits.end()) continue;
      s = tile_candidate_;
    } else {
      if (tuning_on && !fits.empty()) fits.push_back(kUnfused);
      s = S.shape_for(A->key, fits, tuning_on, &tuning);
      if (s < 0 || (s == kUnfused && !tuning)) continue;
    }
    if (trace) FusionPlanner::trace(q, *A, *this);
    FusedItem it;
    it.first = A->first;
    it.n = A->n;
    it.tuning = tuning;
    it.unfused = s == kUnfused;
    it.key = A->key;
    it.shape = s;
    // timing name: the group and the chain's first and last compute kernels
    std::string k0, k1;
    for (size_t l = 0; l < A->n; l++)
      if (!A->loops[l].copy) {
        const std::string &kn = q[A->first + l].loop->kernel;
        const std::string shortname = kn.substr(kn.find('/') + 1);
        if (k0.empty()) k0 = shortname;
        k1 = shortname;
      }
    it.name = std::string("fused/") + G.name + "[" + k0 + ".." + k1 + "]";
    it.bytes = A->fused_bytes;
    it.loop_bytes = A->loop_bytes;
    it.launch = G.launch;
    it.analysis = A;
    items.push_back(std::move(it));
  }
}

// The device plan of a chosen chain, built when the planner reaches it in
// queue order: renamed dats move to their shadow storage now, so the loops
// planned after it see the new storage and those before it the old.
void Runtime::build_fused(const std::vector<Desc> &q, FusedItem &it) {
  FusionState &S = fusion_state();
  if (it.shape == kUnfused) {  // timing the unfused loops: the planner brackets them with the events
    it.ev0 = S.event();
    it.ev1 = S.event();
    S.tune[it.key].pending.push_back({it.shape, {it.ev0, it.ev1}});
    return;
  }
  FusionPlanner fp(*this);
  const ChainAnalysis &A = *std::static_pointer_cast<ChainAnalysis>(it.analysis);
  auto plan = std::make_unique<FPlan>();
  fp.build(q, A, cand_shape(it.shape).tx, cand_shape(it.shape).ty, cand_stage_ro(it.shape), *plan, it.renamed);
  plan->red_counter = red_counters_ + (A.first % kNumCounters);
  it.smem = plan->smem_doubles * 8;
  const int occ = S.occupancy.at({A.group, it.smem});
  it.grid = (int)std::min<long long>((long long)plan->ntx * plan->nty, 148LL * occ);
  // the device copy of this plan (identical plans share one)
  uint64_t ph = 0xCBF29CE484222325ULL;
  const unsigned char *pb = reinterpret_cast<const unsigned char *>(plan.get());
  for (size_t k = 0; k < sizeof(FPlan); k++) ph = (ph ^ pb[k]) * 0x100000001B3ULL;
  auto pit = S.plans.find(ph);
  if (pit == S.plans.end()) {
    FPlan *dp = nullptr;
    OPSB_CUDA(cudaMalloc(&dp, sizeof(FPlan)));
    OPSB_CUDA(cudaMemcpyAsync(dp, plan.get(), sizeof(FPlan), cudaMemcpyHostToDevice, stream_));
    pit = S.plans.emplace(ph, std::make_pair(dp, std::move(plan))).first;
  }
  it.dplan = pit->second.first;
  if (it.tuning) {
    it.ev0 = S.event();
    it.ev1 = S.event();
    S.tune[A.key].pending.push_back({it.shape, {it.ev0, it.ev1}});
  }
}

}  // namespace opsb
