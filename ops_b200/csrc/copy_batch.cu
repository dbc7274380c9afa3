// Batched execution of boundary-copy loops.
//
// The reference apps refresh their reflective boundaries with dozens of thin
// loops per call (CloverLeaf 2D update_halo.cpp queues up to 40, the 3D app
// up to 84), each copying (or negating) a strip of halo cells from a mirror
// point inside the domain. One launch each leaves the GPU idle between
// launches of a few microseconds of work. A run of such loops in the queue
// (kernels registered with a CopyLoopSpec) is executed instead as a few
// launches of one copy kernel over a list of strips: every (loop, field)
// pair becomes a strip; a strip goes into the first batch after every
// earlier strip it conflicts with (same dat, and its write box meets the
// other's write or read box, or its read box meets the other's write box),
// so batches hold only independent strips and keep the queue's order where
// it matters. Each strip checks its field flag on the device (the flags are
// this flush's staged globals), so the batches depend only on the queue's
// structure and stay valid when a captured graph replays them with other
// flags. The values moved are the same doubles the loops would move: the
// results are identical.
#include <cstring>
#include <unordered_map>

#include "runtime.h"

namespace opsb {

namespace {
std::map<std::string, CopyLoopSpec> &copy_specs() {
  static std::map<std::string, CopyLoopSpec> m;
  return m;
}
std::unordered_map<const LoopInfo *, const CopyLoopSpec *> &copy_spec_cache() {
  static std::unordered_map<const LoopInfo *, const CopyLoopSpec *> m;
  return m;
}

struct CopyStrip {
  double *p;          // logical origin of the dat
  const int *flag;    // device flag word, or nullptr (always copy)
  long long src;      // element offset of the mirror point
  long long pitch, plane;
  int x0, y0, z0, nx, ny, nz;
  long long first;    // first cell number of this strip in its batch
  int neg, pad;
};

// A batch is cut into chunks of kChunk cells of one strip each (the chunk
// table follows the strips in the same device buffer); a CTA takes a chunk,
// so it finds its strip with one load instead of a search per cell, and
// the cell's (x, y, z) comes from 32-bit arithmetic.
constexpr int kChunk = 1024;
struct Chunk {
  int strip, first;  // strip index, first cell of the chunk within the strip
};

__global__ void copy_batch_kernel(const CopyStrip *__restrict__ s, const Chunk *__restrict__ chunks, int nchunks) {
  for (int c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const Chunk ch = chunks[c];
    const CopyStrip &e = s[ch.strip];
    if (e.flag && *e.flag != 1) continue;  // the same for the whole CTA
    const int nx = e.nx, ny = e.ny;
    const int end = min(ch.first + kChunk, nx * ny * e.nz);
    double *const base = e.p + (long long)e.x0 + (long long)e.y0 * e.pitch + (long long)e.z0 * e.plane;
    for (int k = ch.first + (int)threadIdx.x; k < end; k += blockDim.x) {
      const int r = k / nx, x = k - r * nx;
      const int z = r / ny, y = r - z * ny;
      double *q = base + x + (long long)y * e.pitch + (long long)z * e.plane;
      const double v = q[e.src];
      *q = e.neg ? -v : v;
    }
  }
}

struct Box {
  int lo[3], hi[3];  // inclusive
};
bool meet(const Box &a, const Box &b) {
  for (int k = 0; k < 3; k++)
    if (a.hi[k] < b.lo[k] || b.hi[k] < a.lo[k]) return false;
  return true;
}

struct Planned {
  std::vector<std::vector<CopyStrip>> batches;
  long long cells = 0;
};

// Strips of queue items [i, i + n) grouped into batches (see the file comment).
bool plan(const std::vector<Desc> &q, size_t i, int n, Planned &out) {
  Runtime &rt = Runtime::get();
  struct Item { CopyStrip s; Box w, r; const char *data; int batch; };
  std::vector<Item> items;
  for (int j = 0; j < n; j++) {
    const Desc &d = q[i + j];
    const CopyLoopSpec *sp = find_copy_loop(d.loop);
    if (!sp) return false;
    const int *flags = nullptr;
    if (sp->flags_arg >= 0) flags = reinterpret_cast<const int *>(rt.gbl_device() + d.gbl_off[sp->flags_arg]);
    for (int f = 0; f < sp->nfields; f++) {
      const Arg &a = d.args[sp->arg[f]];
      Dat &dt = rt.dat(a.dat);
      if (dt.elem_size != 8 || rt.stencil(a.stencil).type != 0) return false;
      Item it;
      CopyStrip &s = it.s;
      s.p = reinterpret_cast<double *>(dt.origin_ptr());
      s.flag = flags ? flags + sp->flag[f] : nullptr;
      s.pitch = dt.pitch;
      s.plane = dt.plane;
      s.src = sp->off[0] + sp->off[1] * dt.pitch + sp->off[2] * dt.plane;
      s.x0 = d.range[0]; s.y0 = d.range[2]; s.z0 = d.range[4];
      s.nx = d.range[1] - d.range[0]; s.ny = d.range[3] - d.range[2]; s.nz = d.range[5] - d.range[4];
      s.neg = sp->neg;
      s.pad = 0;
      if (s.nx <= 0 || s.ny <= 0 || s.nz <= 0) continue;
      for (int k = 0; k < 3; k++) {
        it.w.lo[k] = d.range[2 * k];
        it.w.hi[k] = d.range[2 * k + 1] - 1;
        it.r.lo[k] = it.w.lo[k] + sp->off[k];
        it.r.hi[k] = it.w.hi[k] + sp->off[k];
      }
      if (meet(it.w, it.r)) return false;  // a strip reading its own cells: keep the loop
      it.data = dt.data_d;
      it.batch = 0;
      for (const Item &e : items)
        if (e.data == it.data && e.batch >= it.batch && (meet(it.w, e.w) || meet(it.w, e.r) || meet(it.r, e.w)))
          it.batch = e.batch + 1;
      items.push_back(it);
    }
  }
  int nb = 0;
  for (const Item &e : items) nb = std::max(nb, e.batch + 1);
  out.batches.assign(nb, {});
  out.cells = 0;
  for (Item &e : items) {
    std::vector<CopyStrip> &b = out.batches[e.batch];
    long long first = b.empty() ? 0 : b.back().first + (long long)b.back().nx * b.back().ny * b.back().nz;
    e.s.first = first;
    b.push_back(e.s);
    out.cells += (long long)e.s.nx * e.s.ny * e.s.nz;
  }
  return true;
}

// Device copies of strip lists and their chunk tables, kept by content: a
// captured graph keeps pointing at them, so they are never rewritten or freed.
std::unordered_map<uint64_t, CopyStrip *> &strip_cache() {
  static std::unordered_map<uint64_t, CopyStrip *> m;
  return m;
}
uint64_t hash_bytes(const void *p, size_t n) {
  const unsigned char *c = static_cast<const unsigned char *>(p);
  uint64_t h = 0xCBF29CE484222325ULL;
  for (size_t k = 0; k < n; k++) h = (h ^ c[k]) * 0x100000001B3ULL;
  return h ^ n;
}
// The batch's chunks: every strip cut into runs of kChunk cells.
std::vector<Chunk> chunks_of(const std::vector<CopyStrip> &b) {
  std::vector<Chunk> ch;
  for (size_t i = 0; i < b.size(); i++) {
    const long long cells = (long long)b[i].nx * b[i].ny * b[i].nz;
    if (cells >= (1LL << 31) - kChunk) throw Error(E_UNSUPPORTED, "copy batch: strip of 2^31 cells or more");
    for (long long f = 0; f < cells; f += kChunk) ch.push_back({(int)i, (int)f});
  }
  return ch;
}
// One buffer: the strips, then (16-byte aligned) the chunk table.
CopyStrip *device_strips(const std::vector<CopyStrip> &b, const std::vector<Chunk> &ch, bool may_upload) {
  const size_t sbytes = (b.size() * sizeof(CopyStrip) + 15) / 16 * 16;
  std::vector<unsigned char> blob(sbytes + ch.size() * sizeof(Chunk), 0);
  memcpy(blob.data(), b.data(), b.size() * sizeof(CopyStrip));
  if (!ch.empty()) memcpy(blob.data() + sbytes, ch.data(), ch.size() * sizeof(Chunk));
  const uint64_t h = hash_bytes(blob.data(), blob.size());
  auto it = strip_cache().find(h);
  if (it != strip_cache().end()) return it->second;
  if (!may_upload) return nullptr;
  CopyStrip *d = nullptr;
  OPSB_CUDA(cudaMalloc(&d, blob.size()));
  // ordered before the batch's launch on the same stream; the pageable
  // source is staged before the call returns
  OPSB_CUDA(cudaMemcpyAsync(d, blob.data(), blob.size(), cudaMemcpyHostToDevice, Runtime::get().stream()));
  strip_cache()[h] = d;
  return d;
}


int match_copy_run(const std::vector<Desc> &q, size_t i) {
  size_t j = i;
  while (j < q.size() && !q[j].loop->internal && find_copy_loop(q[j].loop)) j++;
  int n = (int)(j - i);
  if (n < 2) return 0;
  Planned pl;
  if (!plan(q, i, n, pl)) return 0;
  return n;
}

// Planned before any capture: the strips are uploaded now (once per
// distinct strip list) and the launches keep their device addresses.
PlanItem prepare_copy_run(const std::vector<Desc> &q, size_t i, int n) {
  Planned pl;
  if (!plan(q, i, n, pl)) throw Error(E_STATE, "copy batch: plan failed after a match");
  struct Launch { CopyStrip *d; const Chunk *ch; int nchunks; int blocks; };
  std::vector<Launch> ls;
  for (const auto &b : pl.batches) {
    if (b.empty()) continue;
    const std::vector<Chunk> ch = chunks_of(b);
    if (ch.empty()) continue;
    CopyStrip *d = device_strips(b, ch, true);
    const size_t sbytes = (b.size() * sizeof(CopyStrip) + 15) / 16 * 16;
    const Chunk *dch = reinterpret_cast<const Chunk *>(reinterpret_cast<const char *>(d) + sbytes);
    const int blocks = (int)std::min<size_t>(ch.size(), 148 * 8);
    ls.push_back({d, dch, (int)ch.size(), blocks});
  }
  PlanItem it;
  it.name = "runtime/copy_batch";
  it.kernels = (long long)ls.size();
  it.bytes = 16.0 * (double)pl.cells;
  if (!ls.empty())
    it.run = [ls](cudaStream_t s) {
      for (const Launch &l : ls) {
        copy_batch_kernel<<<l.blocks, 256, 0, s>>>(l.d, l.ch, l.nchunks);
        OPSB_CUDA(cudaGetLastError());
      }
    };
  return it;
}

struct CopyChainReg {
  CopyChainReg() {
    ChainRule r;
    r.name = "runtime/copy_batch";
    r.match = match_copy_run;
    r.prepare = prepare_copy_run;
    Runtime::register_chain(r);
  }
};
CopyChainReg copy_chain_reg;
}  // namespace

void register_copy_loop(const std::string &kernel, const CopyLoopSpec &spec) { copy_specs()[kernel] = spec; }

const CopyLoopSpec *find_copy_loop(const LoopInfo *loop) {
  auto &c = copy_spec_cache();
  auto it = c.find(loop);
  if (it != c.end()) return it->second;
  auto f = copy_specs().find(loop->kernel);
  const CopyLoopSpec *sp = f == copy_specs().end() ? nullptr : &f->second;
  c[loop] = sp;
  return sp;
}

}  // namespace opsb
