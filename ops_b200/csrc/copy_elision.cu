// Copy elision by renaming (a lazy-queue rewrite).
//
// A pure copy loop  dst(0,0) = src(0,0)  over a range R, followed in the same
// flush by a loop W that overwrites src over exactly R (WRITE access, centre
// point only) without reading it, leaves src's old interior dead. Instead of
// moving R's cells, the two dats exchange their device storage and then swap
// back the cells OUTSIDE R (halos and any margin), which the copy would not
// have touched. The result is identical to the copy, while HBM traffic drops
// from a read and a write of R to a read and a write of the (small)
// complement of R. Laplace's  copy(A <- Anew); apply_stencil(A -> Anew)
// (apps/c/laplace2d_tutorial/step7/laplace2d.cpp:116-124) is the case this
// targets: each iteration then moves 16 bytes per cell instead of 32.
#include <algorithm>

#include "runtime.h"

namespace opsb {

namespace {
struct Box {
  int lo[3], hi[3];
};
struct SwapParams {
  char *a, *b;           // storage bases of the two dats (same layout)
  long long origin;      // element offset of logical (0,0,0)
  long long pitch, plane;
  int elem;              // bytes per point
  int nbox;
  long long prefix[7];   // cumulative cell counts per box
  Box box[6];
};

__global__ void swap_outside_kernel(const __grid_constant__ SwapParams p) {
  const long long total = p.prefix[p.nbox];
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    int b = 0;
    while (c >= p.prefix[b + 1]) b++;
    const Box &bx = p.box[b];
    long long r = c - p.prefix[b];
    const int nx = bx.hi[0] - bx.lo[0];
    const int ny = bx.hi[1] - bx.lo[1];
    const int x = bx.lo[0] + (int)(r % nx);
    r /= nx;
    const int y = bx.lo[1] + (int)(r % ny);
    const int z = bx.lo[2] + (int)(r / ny);
    const long long off = (p.origin + x + (long long)y * p.pitch + (long long)z * p.plane) * p.elem;
    if (p.elem == 8) {
      double *pa = reinterpret_cast<double *>(p.a + off), *pb = reinterpret_cast<double *>(p.b + off);
      double t = *pa; *pa = *pb; *pb = t;
    } else {
      for (int k = 0; k < p.elem; k++) {
        char t = p.a[off + k]; p.a[off + k] = p.b[off + k]; p.b[off + k] = t;
      }
    }
  }
}

LoopInfo &swap_outside_info() {
  static LoopInfo li = [] {
    LoopInfo l;
    l.kernel = "__swap_outside";
    l.nparams = 2;
    l.internal = 1;
    return l;
  }();
  return li;
}

bool zero_point_stencil(const Stencil &s) {
  if (s.points != 1 || s.type != 0) return false;
  for (int v : s.offs)
    if (v != 0) return false;
  return true;
}
}  // namespace

PlanItem Runtime::prepare_swap_outside(const Desc &d) {
  const Dat &A = *dats_[d.args[0].dat];
  const Dat &B = *dats_[d.args[1].dat];
  SwapParams p;
  memset(&p, 0, sizeof(p));
  p.a = A.data_d;
  p.b = B.data_d;
  p.origin = A.origin;
  p.pitch = A.pitch;
  p.plane = A.plane;
  p.elem = A.elem_size;
  const int nd = d.dim;
  int elo[3], ehi[3], rlo[3], rhi[3];
  for (int i = 0; i < 3; i++) {
    if (i < nd) {
      elo[i] = A.lo[i];  // the stored window
      ehi[i] = A.hi[i];
      rlo[i] = std::max(d.range[2 * i], elo[i]);
      rhi[i] = std::min(d.range[2 * i + 1], ehi[i]);
    } else {
      elo[i] = rlo[i] = 0;
      ehi[i] = rhi[i] = 1;
    }
  }
  // Complement of R in the extent: for each dimension k (outermost first),
  // the slabs below and above R along k, with outer dims restricted to R and
  // inner dims spanning the full extent.
  int nb = 0;
  for (int k = nd - 1; k >= 0; k--) {
    for (int side = 0; side < 2; side++) {
      Box b;
      for (int i = 0; i < 3; i++) {
        if (i > k) { b.lo[i] = rlo[i]; b.hi[i] = rhi[i]; }
        else if (i < k) { b.lo[i] = elo[i]; b.hi[i] = ehi[i]; }
        else if (side == 0) { b.lo[i] = elo[i]; b.hi[i] = rlo[i]; }
        else { b.lo[i] = rhi[i]; b.hi[i] = ehi[i]; }
      }
      long long n = 1;
      for (int i = 0; i < 3; i++) n *= std::max(0, b.hi[i] - b.lo[i]);
      if (n > 0) p.box[nb++] = b;
    }
  }
  p.nbox = nb;
  p.prefix[0] = 0;
  for (int i = 0; i < nb; i++) {
    long long n = 1;
    for (int k = 0; k < 3; k++) n *= (p.box[i].hi[k] - p.box[i].lo[k]);
    p.prefix[i + 1] = p.prefix[i] + n;
  }
  PlanItem it;
  it.name = d.loop->kernel;
  if (nb == 0) return it;
  long long total = p.prefix[nb];
  int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 8);
  it.kernels = 1;
  it.run = [p, blocks](cudaStream_t s) {
    swap_outside_kernel<<<blocks, 256, 0, s>>>(p);
    OPSB_CUDA(cudaGetLastError());
  };
  return it;
}

void Runtime::elide_copies(std::vector<Desc> &q) {
  if (!fusion_on_) return;
  for (size_t i = 0; i < q.size(); i++) {
    Desc &c = q[i];
    if (c.loop->internal || c.loop->copy_dst < 0) continue;
    const Arg &ad = c.args[c.loop->copy_dst];
    const Arg &as = c.args[c.loop->copy_src];
    if (!ad.opt || !as.opt || ad.kind != ARG_DAT || as.kind != ARG_DAT || ad.dat == as.dat) continue;
    if (!zero_point_stencil(stencils_[ad.stencil]) || !zero_point_stencil(stencils_[as.stencil])) continue;
    Dat &D = *dats_[ad.dat];
    Dat &S = *dats_[as.dat];
    if (D.bytes != S.bytes || D.pitch != S.pitch || D.origin != S.origin || D.elem_size != S.elem_size ||
        D.dim != S.dim || D.locked || S.locked)
      continue;
    bool same_extent = true;
    for (int k = 0; k < 3; k++)
      same_extent &= (D.size[k] == S.size[k] && D.d_m[k] == S.d_m[k] && D.base[k] == S.base[k] &&
                      D.lo[k] == S.lo[k] && D.hi[k] == S.hi[k]);
    if (!same_extent) continue;
    // Earlier loops of this flush must not see the renamed storage.
    bool earlier = false;
    for (size_t j = 0; j < i && !earlier; j++)
      for (const Arg &a : q[j].args)
        if (a.kind == ARG_DAT && (a.dat == D.index || a.dat == S.index)) earlier = true;
    if (earlier) continue;
    // The next loop touching src must overwrite exactly R without reading src.
    bool ok = false;
    for (size_t j = i + 1; j < q.size(); j++) {
      const Desc &w = q[j];
      int refs = 0, good = 0;
      for (const Arg &a : w.args) {
        if (a.kind != ARG_DAT || a.dat != S.index) continue;
        refs++;
        if (a.opt && a.acc == ACC_WRITE && zero_point_stencil(stencils_[a.stencil])) good++;
      }
      if (refs == 0) continue;
      bool same_range = true;
      for (int k = 0; k < 6; k++) same_range &= (w.range[k] == c.range[k]);
      ok = (refs == 1 && good == 1 && same_range && !w.loop->internal);
      break;
    }
    if (!ok) continue;
    // Rename: dst takes src's storage, src takes dst's; then the cells outside
    // R are swapped back so both keep their own halos.
    std::swap(D.data_d, S.data_d);
    D.host.clear();
    S.host.clear();
    Desc x;
    x.loop = &swap_outside_info();
    x.name = "__swap_outside";
    x.block = c.block;
    x.dim = c.dim;
    memcpy(x.range, c.range, sizeof(x.range));
    Arg a0; a0.kind = ARG_DAT; a0.dat = D.index; a0.stencil = ad.stencil;
    Arg a1; a1.kind = ARG_DAT; a1.dat = S.index; a1.stencil = as.stencil;
    x.args = {a0, a1};
    x.red_first = {0, 0};
    x.gbl_off = {0, 0};
    q[i] = std::move(x);
  }
}

}  // namespace opsb
