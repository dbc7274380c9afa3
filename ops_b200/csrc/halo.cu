// Single-process halo transfer between dats of (possibly different) blocks:
// ops_decl_halo / ops_decl_halo_group / ops_halo_transfer
// (ops/c/src/core/ops_lib_core.cpp:998-1040,
// ops/c/src/core/ops_device_singlenode_common.cpp:262-346). The reference
// packs each halo's source box into a linear buffer and unpacks it into the
// target with two kernels per halo; here one kernel walks the iteration box
// of every halo of a group (a work list, one thread per element) and copies
// source to target directly, so a group is one launch and no buffer.
//
// Index rule: dat dimension i walks dimension |dir_i| - 1 of the iteration
// box, backwards when dir_i < 0, starting at logical index base_i; a float
// <-> double pair converts through the narrower type as the reference's
// mixed exchange does.
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "runtime.h"

namespace opsb {
namespace {

struct HaloDev {
  char *src, *dst;                   // logical index (0, 0, 0) of each dat
  long long sst[3], dst_[3];         // element strides per dat dimension
  int n[3], fb[3], tb[3], fd[3], td[3];
  int selem, delem, ncomp, conv;     // conv: 0 bytes, 1 double -> float, 2 float -> double
  long long first, count;
};

__device__ __forceinline__ long long box_offset(const int (&n)[3], const int (&base)[3], const int (&dir)[3],
                                                const long long (&st)[3], const int (&b)[3]) {
  long long off = 0;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const int bd = abs(dir[i]) - 1;
    const int j = dir[i] > 0 ? b[bd] : n[bd] - 1 - b[bd];
    off += (long long)(base[i] + j) * st[i];
  }
  return off;
}

__global__ void k_halo(const HaloDev *__restrict__ hs, int nh, long long total) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    int h = 0;
    while (h + 1 < nh && t >= hs[h + 1].first) h++;
    const HaloDev &d = hs[h];
    long long k = t - d.first;
    int b[3];
    b[0] = (int)(k % d.n[0]);
    k /= d.n[0];
    b[1] = (int)(k % d.n[1]);
    b[2] = (int)(k / d.n[1]);
    const char *s = d.src + box_offset(d.n, d.fb, d.fd, d.sst, b) * d.selem;
    char *o = d.dst + box_offset(d.n, d.tb, d.td, d.dst_, b) * d.delem;
    if (d.conv == 1) {
      for (int c = 0; c < d.ncomp; c++) reinterpret_cast<float *>(o)[c] = (float)reinterpret_cast<const double *>(s)[c];
    } else if (d.conv == 2) {
      for (int c = 0; c < d.ncomp; c++) reinterpret_cast<double *>(o)[c] = (double)reinterpret_cast<const float *>(s)[c];
    } else if ((d.selem & 7) == 0) {
      for (int c = 0; c < d.selem / 8; c++) reinterpret_cast<long long *>(o)[c] = reinterpret_cast<const long long *>(s)[c];
    } else if ((d.selem & 3) == 0) {
      for (int c = 0; c < d.selem / 4; c++) reinterpret_cast<int *>(o)[c] = reinterpret_cast<const int *>(s)[c];
    } else {
      for (int c = 0; c < d.selem; c++) o[c] = s[c];
    }
  }
}

bool is_float_type(const std::string &t) { return t == "double" || t == "float"; }

// A checked condition whose message is built only when the check fails.
#define HALO_REQUIRE(cond, code, msg)        \
  do {                                       \
    if (!(cond)) throw Error((code), (msg)); \
  } while (0)

}  // namespace

int Runtime::decl_halo(int from, int to, const int *iter, const int *from_base, const int *to_base,
                       const int *from_dir, const int *to_dir) {
  HALO_REQUIRE(inited_, E_STATE, "ops_decl_halo before ops_init");
  HALO_REQUIRE(iter && from_base && to_base && from_dir && to_dir, E_ARG, "ops_decl_halo: null array");
  Dat &f = dat(from);
  Dat &t = dat(to);
  const int dims = blocks_[f.block].dims;
  HALO_REQUIRE(blocks_[t.block].dims == dims, E_ARG, "ops_decl_halo: the two dats' blocks differ in dimension");
  HALO_REQUIRE(f.dim == t.dim, E_ARG, "ops_decl_halo: the two dats differ in components per point");
  if (f.type != t.type || f.type_size != t.type_size)
    HALO_REQUIRE(is_float_type(f.type) && is_float_type(t.type), E_UNSUPPORTED,
            "ops_decl_halo: a mixed exchange is supported between float and double only");
  Halo h;
  h.from = from;
  h.to = to;
  for (int i = 0; i < 3; i++) {
    const bool real = i < dims;
    h.iter[i] = real ? iter[i] : 1;
    h.fbase[i] = real ? from_base[i] : 0;
    h.tbase[i] = real ? to_base[i] : 0;
    h.fdir[i] = real ? from_dir[i] : i + 1;
    h.tdir[i] = real ? to_dir[i] : i + 1;
    HALO_REQUIRE(h.iter[i] >= 0, E_ARG, "ops_decl_halo: negative iteration size");
  }
  // directions: a permutation of +-1..dims for each side
  for (int side = 0; side < 2; side++) {
    const int *dir = side ? h.tdir : h.fdir;
    int seen = 0;
    for (int i = 0; i < dims; i++) {
      const int a = std::abs(dir[i]);
      HALO_REQUIRE(a >= 1 && a <= dims && !(seen & (1 << a)), E_ARG, "ops_decl_halo: directions must permute +-1..dims");
      seen |= 1 << a;
    }
  }
  // both boxes inside the dats' allocations (no device access can leave them)
  for (int side = 0; side < 2; side++) {
    const Dat &d = side ? t : f;
    const int *base = side ? h.tbase : h.fbase;
    const int *dir = side ? h.tdir : h.fdir;
    for (int i = 0; i < dims; i++) {
      const int n = h.iter[std::abs(dir[i]) - 1];
      if (n == 0) continue;
      const int lo = d.lo[i], hi = d.hi[i];
      HALO_REQUIRE(base[i] >= lo && base[i] + n <= hi, E_ARG,
              "ops_decl_halo: the box on dat " + d.name + " leaves its allocation in dimension " + std::to_string(i));
    }
  }
  halos_.push_back(h);
  return (int)halos_.size() - 1;
}

int Runtime::decl_halo_group(int n, const int *halos) {
  HALO_REQUIRE(inited_, E_STATE, "ops_decl_halo_group before ops_init");
  HALO_REQUIRE(n >= 0 && (n == 0 || halos), E_ARG, "ops_decl_halo_group: bad list");
  std::vector<int> g;
  for (int i = 0; i < n; i++) {
    HALO_REQUIRE(halos[i] >= 0 && halos[i] < (int)halos_.size(), E_ARG, "ops_decl_halo_group: unknown halo");
    g.push_back(halos[i]);
  }
  halo_groups_.push_back(g);
  return (int)halo_groups_.size() - 1;
}

void Runtime::halo_transfer(int group) {
  HALO_REQUIRE(group >= 0 && group < (int)halo_groups_.size(), E_ARG, "ops_halo_transfer: unknown group");
  const std::vector<int> &g = halo_groups_[group];
  if (g.empty()) return;
  execute();  // loops queued before the transfer see the old halos, loops after it the new ones
  std::vector<HaloDev> descs;
  for (int hi : g) {
    const Halo &h = halos_[hi];
    const Dat &f = dat(h.from);
    const Dat &t = dat(h.to);
    HALO_REQUIRE(f.locked == 0 && t.locked == 0, E_STATE, "ops_halo_transfer on a dat whose raw pointer is held");
    HALO_REQUIRE(f.split < 0 && t.split < 0, E_UNSUPPORTED,
                 "ops_halo_transfer between dats partitioned across ranks is not supported");
    HaloDev d;
    memset(&d, 0, sizeof(d));
    d.src = f.origin_ptr();
    d.dst = t.origin_ptr();
    const long long fs[3] = {1, f.pitch, f.plane}, ts[3] = {1, t.pitch, t.plane};
    for (int i = 0; i < 3; i++) {
      d.sst[i] = fs[i];
      d.dst_[i] = ts[i];
      d.n[i] = h.iter[i];
      d.fb[i] = h.fbase[i];
      d.tb[i] = h.tbase[i];
      d.fd[i] = h.fdir[i];
      d.td[i] = h.tdir[i];
    }
    d.selem = f.elem_size;
    d.delem = t.elem_size;
    d.ncomp = f.dim;
    d.conv = f.type_size == t.type_size ? 0 : (f.type_size == 8 ? 1 : 2);
    d.count = (long long)h.iter[0] * h.iter[1] * h.iter[2];
    if (d.count > 0) descs.push_back(d);
  }
  if (descs.empty()) return;
  // One launch when the halos are independent (no dat written twice, none
  // both read and written); otherwise one launch per halo in declaration
  // order, as the reference applies them.
  bool independent = true;
  for (size_t i = 0; i < g.size() && independent; i++)
    for (size_t j = 0; j < g.size(); j++) {
      const Halo &a = halos_[g[i]], &b = halos_[g[j]];
      if ((i != j && a.to == b.to) || a.to == b.from) {
        independent = false;
        break;
      }
    }
  const size_t need = descs.size() * sizeof(HaloDev);
  if (need > halo_desc_cap_) {
    if (halo_desc_d_) cudaFree(halo_desc_d_);
    halo_desc_d_ = nullptr;
    halo_desc_cap_ = std::max<size_t>(need, 64 * sizeof(HaloDev));
    OPSB_CUDA(cudaMalloc(&halo_desc_d_, halo_desc_cap_));
  }
  auto launch = [&](size_t first, size_t n) {
    long long total = 0;
    for (size_t k = first; k < first + n; k++) {
      descs[k].first = total;
      total += descs[k].count;
    }
    HaloDev *dev = reinterpret_cast<HaloDev *>(halo_desc_d_) + first;
    OPSB_CUDA(cudaMemcpyAsync(dev, descs.data() + first, n * sizeof(HaloDev), cudaMemcpyHostToDevice, stream_));
    const long long blocks = std::min<long long>((total + 255) / 256, 148LL * 16);
    k_halo<<<(unsigned)blocks, 256, 0, stream_>>>(dev, (int)n, total);
    OPSB_CUDA(cudaGetLastError());
    count_kernels(1);
  };
  if (independent) {
    launch(0, descs.size());
  } else {
    for (size_t k = 0; k < descs.size(); k++) launch(k, 1);
  }
  // the descriptors are read from pageable host memory by the copies above:
  // finish before they go out of scope
  OPSB_CUDA(cudaStreamSynchronize(stream_));
}

}  // namespace opsb
