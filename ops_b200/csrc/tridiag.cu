// Batched tridiagonal solver (ops_tridMultiDimBatch / _Inc).
//
// Reference: ops/c/src/tridiag/ops_tridiag.cpp:78-249 hands every line along
// `solvedim` of the range to the external Tridsolver library
// (trid{D,S}mtsvStridedBatch[Inc]); each line is the system
//     a_i x_{i-1} + b_i x_i + c_i x_{i+1} = d_i   (a_0, c_{n-1} unused).
// The non-Inc form overwrites d with x; the Inc form adds x to u.
//
// B200 design: one persistent launch walks a work list of line groups over
// any number of systems (blocks of different shapes solve in one launch).
// Every line is split into chunks, one chunk per thread; a thread runs the
// modified Thomas elimination on its chunk in registers, expressing each row
// through the chunk's first and last unknowns (the partition method of
// Wang 1981, as used for GPUs by Laszlo, Giles and Appleyard, ACM TOMS 42(4)
// 2016). The chunks' end rows form a small tridiagonal system in shared
// memory, solved by Thomas; a last pass substitutes back. Coefficients and
// right-hand sides are read once and the solution written once: 40 bytes per
// FP64 unknown (48 for _Inc), nothing else touches HBM.
//   * lines along y or z (strided): a warp holds 32 neighbouring lines
//     (coalesced along x), the 8 warps of a CTA hold the 8 chunks;
//   * lines along x (contiguous): a warp holds one line, lane = chunk.
#include <algorithm>
#include <cstdio>
#include <vector>

#include "../../include/ops_b200.h"
#include "runtime.h"

namespace opsb {
namespace trid {

struct Sys {
  const char *a, *b, *c;
  char *d, *u;
  int n;           // line length
  int nl0, nl1;    // line counts along the two non-solve dimensions (fastest first)
  long long ss;    // stride along the solve dimension (elements)
  long long s0, s1;
};

struct Work {
  int sys, l0, l1;  // system, first line along dim 0, line index along dim 1
};

// Reciprocal by Newton-Raphson refinement (Newton's method for 1/x,
// e = 1 - x r, r' = r + r e, which doubles the correct bits per step) from a
// hardware approximation. It is accurate to about 1 ulp without the
// out-of-line slow path of IEEE division, whose call would force the
// per-thread coefficient arrays out of registers. Valid for finite normal
// pivots with 2^-1000 < |x| < 2^1000; the solver's tolerance is relative
// (1e-12 in FP64), not bit-exact.
__device__ __forceinline__ float recip(float x) {
  float r = __fdividef(1.0f, x);
  const float e = fmaf(-x, r, 1.0f);
  return fmaf(r, e, r);
}
__device__ __forceinline__ double recip(double x) {
  // Scale x to [1, 2) by its exponent so the single-precision seed never
  // over- or underflows, refine twice, then undo the scaling.
  const long long bits = __double_as_longlong(x);
  const long long ex = (bits >> 52) & 0x7ff;
  const double m = __longlong_as_double((bits & ~(0x7ffLL << 52)) | (1023LL << 52));
  double r = (double)__fdividef(1.0f, (float)m);
  double e = fma(-m, r, 1.0);
  r = fma(r, e, r);
  e = fma(-m, r, 1.0);
  r = fma(r, e, r);
  return r * __longlong_as_double((2046LL - ex) << 52);
}

// Modified Thomas on rows [r0, r0+m) of one line (m >= 2): afterwards row i
// reads  aa_i x_first + x_i + cc_i x_last = dd_i  for 0 < i < m-1, and the
// end rows keep their outside couplings:
//   aa_0 x_prev_last + x_first + cc_0 x_last   = dd_0
//   aa_{m-1} x_first + x_last + cc_{m-1} x_next_first = dd_{m-1}
// The last row's coefficients are returned in la, lc, ld as they are
// produced (row m-1 is final after the forward sweep); reading them back
// from the arrays with a run-time index would move the arrays to local memory.
template <class T, int M>
__device__ __forceinline__ void chunk_eliminate(const T *a, const T *b, const T *c, const T *d, long long ss, int m,
                                                T (&aa)[M], T (&cc)[M], T (&dd)[M], T &la, T &lc, T &ld) {
  // All of the chunk's loads are issued before any arithmetic, so each
  // thread keeps 4*m independent requests in flight.
  T bb[M];
#pragma unroll
  for (int i = 0; i < M; i++) {
    if (i < m) {
      aa[i] = __ldg(a + i * ss);
      bb[i] = __ldg(b + i * ss);
      cc[i] = __ldg(c + i * ss);
      dd[i] = __ldg(d + i * ss);
    }
  }
  // Forward sweep in place: (a_i, c_i, d_i) become (aa_i, cc_i, dd_i).
#pragma unroll
  for (int i = 0; i < M; i++) {
    if (i < m) {
      if (i < 2) {
        const T r = recip(bb[i]);
        aa[i] = aa[i] * r;
        cc[i] = cc[i] * r;
        dd[i] = dd[i] * r;
      } else {
        const T ai = aa[i];
        const T r = recip(bb[i] - ai * cc[i - 1]);
        dd[i] = r * (dd[i] - ai * dd[i - 1]);
        aa[i] = -r * ai * aa[i - 1];
        cc[i] = r * cc[i];
      }
      if (i == m - 1) {
        la = aa[i];
        lc = cc[i];
        ld = dd[i];
      }
    }
  }
#pragma unroll
  for (int i = M - 3; i >= 1; i--) {
    if (i <= m - 3) {
      dd[i] = dd[i] - cc[i] * dd[i + 1];
      aa[i] = aa[i] - cc[i] * aa[i + 1];
      cc[i] = -cc[i] * cc[i + 1];
    }
  }
  if (m > 2) {
    const T r = recip(T(1) - cc[0] * aa[1]);
    dd[0] = r * (dd[0] - cc[0] * dd[1]);
    aa[0] = r * aa[0];
    cc[0] = -r * cc[0] * cc[1];
  }
}

// Thomas on the reduced system held in shared memory: row k has
// A[k] x_{k-1} + x_k + C[k] x_{k+1} = D[k]; the solution overwrites D.
template <class T>
__device__ __forceinline__ void reduced_solve(T *A, T *C, T *D, int n, int stride) {
  // forward
  T cp = C[0];
  T dp = D[0];
  C[0] = cp;
  for (int k = 1; k < n; k++) {
    const T ak = A[k * stride];
    const T r = recip(T(1) - ak * cp);
    cp = C[k * stride] * r;
    dp = (D[k * stride] - ak * dp) * r;
    C[k * stride] = cp;
    D[k * stride] = dp;
  }
  for (int k = n - 2; k >= 0; k--) D[k * stride] = D[k * stride] - C[k * stride] * D[(k + 1) * stride];
}

template <class T, int M>
__device__ __forceinline__ void chunk_store(T *d, T *u, long long ss, int m, const T (&aa)[M], const T (&cc)[M],
                                            const T (&dd)[M], T xf, T xl) {
#pragma unroll
  for (int i = 0; i < M; i++) {
    if (i < m) {
      T x = (i == 0) ? xf : (i == m - 1) ? xl : dd[i] - aa[i] * xf - cc[i] * xl;
      if (u) u[i * ss] += x;
      else d[i * ss] = x;
    }
  }
}

constexpr int kLinesContig = 8;      // warps per CTA = lines per CTA (lane = chunk)

// Lines along y or z: threadIdx.x = line (neighbouring x), threadIdx.y =
// chunk. L lines x K chunks = 256 threads: FP64 uses 16 x 16 so that a chunk
// of a 256-point line (16 rows, three coefficient arrays) stays in registers.
template <class T, int M, int L, int K>
__global__ void __launch_bounds__(256) trid_strided_kernel(const Sys *__restrict__ sys, const Work *__restrict__ work,
                                                           int nwork) {
  __shared__ T A[2 * K][L], C[2 * K][L], Dv[2 * K][L];
  const int lane = threadIdx.x, chunk = threadIdx.y;
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const Work wk = work[w];
    const Sys s = sys[wk.sys];
    const int line = wk.l0 + lane;
    const bool active = line < s.nl0;
    const int n = s.n;
    const int kact = n >= 2 * K ? K : (n / 2 > 0 ? n / 2 : 1);
    const int r0 = chunk * n / kact, r1 = (chunk + 1) * n / kact, m = r1 - r0;
    const long long off = (long long)line * s.s0 + (long long)wk.l1 * s.s1 + (long long)r0 * s.ss;
    const T *a = reinterpret_cast<const T *>(s.a) + off;
    const T *b = reinterpret_cast<const T *>(s.b) + off;
    const T *c = reinterpret_cast<const T *>(s.c) + off;
    T *d = reinterpret_cast<T *>(s.d) + off;
    T *u = s.u ? reinterpret_cast<T *>(s.u) + off : nullptr;
    T aa[M], cc[M], dd[M];
    const bool mine = active && chunk < kact;
    if (mine && n == 1) {
      const T x = __ldg(d) * recip(__ldg(b));
      if (u) *u += x;
      else *d = x;
    }
    const bool work_here = mine && n > 1;
    if (work_here) {
      T la = T(0), lc = T(0), ld = T(0);
      chunk_eliminate<T, M>(a, b, c, d, s.ss, m, aa, cc, dd, la, lc, ld);
      A[2 * chunk][lane] = chunk == 0 ? T(0) : aa[0];
      C[2 * chunk][lane] = cc[0];
      Dv[2 * chunk][lane] = dd[0];
      A[2 * chunk + 1][lane] = la;
      C[2 * chunk + 1][lane] = chunk == kact - 1 ? T(0) : lc;
      Dv[2 * chunk + 1][lane] = ld;
    }
    __syncthreads();
    if (chunk == 0 && active && n > 1) reduced_solve<T>(&A[0][lane], &C[0][lane], &Dv[0][lane], 2 * kact, L);
    __syncthreads();
    if (work_here) chunk_store<T, M>(d, u, s.ss, m, aa, cc, dd, Dv[2 * chunk][lane], Dv[2 * chunk + 1][lane]);
    __syncthreads();
  }
}

// Lines along x: threadIdx.y = line, threadIdx.x = chunk.
template <class T, int M>
__global__ void __launch_bounds__(256) trid_contig_kernel(const Sys *__restrict__ sys, const Work *__restrict__ work,
                                                          int nwork) {
  __shared__ T A[kLinesContig][64], C[kLinesContig][64], Dv[kLinesContig][64];
  const int chunk = threadIdx.x, wl = threadIdx.y;
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const Work wk = work[w];
    const Sys s = sys[wk.sys];
    const int line = wk.l0 + wl;
    const bool active = line < s.nl0;
    const int n = s.n;
    const int kact = n >= 64 ? 32 : (n / 2 > 0 ? n / 2 : 1);
    const int r0 = chunk * n / kact, r1 = (chunk + 1) * n / kact, m = r1 - r0;
    const long long off = (long long)line * s.s0 + (long long)wk.l1 * s.s1 + (long long)r0 * s.ss;
    const T *a = reinterpret_cast<const T *>(s.a) + off;
    const T *b = reinterpret_cast<const T *>(s.b) + off;
    const T *c = reinterpret_cast<const T *>(s.c) + off;
    T *d = reinterpret_cast<T *>(s.d) + off;
    T *u = s.u ? reinterpret_cast<T *>(s.u) + off : nullptr;
    T aa[M], cc[M], dd[M];
    const bool mine = active && chunk < kact;
    if (mine && n == 1) {
      const T x = __ldg(d) * recip(__ldg(b));
      if (u) *u += x;
      else *d = x;
    }
    const bool work_here = mine && n > 1;
    if (work_here) {
      T la = T(0), lc = T(0), ld = T(0);
      chunk_eliminate<T, M>(a, b, c, d, s.ss, m, aa, cc, dd, la, lc, ld);
      A[wl][2 * chunk] = chunk == 0 ? T(0) : aa[0];
      C[wl][2 * chunk] = cc[0];
      Dv[wl][2 * chunk] = dd[0];
      A[wl][2 * chunk + 1] = la;
      C[wl][2 * chunk + 1] = chunk == kact - 1 ? T(0) : lc;
      Dv[wl][2 * chunk + 1] = ld;
    }
    __syncwarp();
    if (chunk == 0 && active && n > 1) reduced_solve<T>(&A[wl][0], &C[wl][0], &Dv[wl][0], 2 * kact, 1);
    __syncwarp();
    if (work_here) chunk_store<T, M>(d, u, s.ss, m, aa, cc, dd, Dv[wl][2 * chunk], Dv[wl][2 * chunk + 1]);
    __syncwarp();
  }
}

// Device copies of the work description, grown as needed.
struct Buffers {
  Sys *sys = nullptr;
  Work *work = nullptr;
  size_t sys_cap = 0, work_cap = 0;
};
Buffers &buffers() {
  static Buffers b;
  return b;
}

template <class T>
void launch(const std::vector<Sys> &systems, int solvedim, cudaStream_t stream, long long *kernels) {
  int maxn = 0;
  for (const Sys &s : systems) maxn = std::max(maxn, s.n);
  if (maxn == 0) return;
  const bool contig = solvedim == 0;
  std::vector<Work> work;
  for (int i = 0; i < (int)systems.size(); i++) {
    const Sys &s = systems[i];
    if (s.n == 0) continue;
    const int g = contig ? kLinesContig : 16;
    for (int l1 = 0; l1 < s.nl1; l1++)
      for (int l0 = 0; l0 < s.nl0; l0 += g) work.push_back({i, l0, l1});
  }
  if (work.empty()) return;
  Buffers &B = buffers();
  if (B.sys_cap < systems.size()) {
    if (B.sys) cudaFree(B.sys);
    B.sys_cap = std::max<size_t>(systems.size(), 64);
    OPSB_CUDA(cudaMalloc(&B.sys, B.sys_cap * sizeof(Sys)));
  }
  if (B.work_cap < work.size()) {
    if (B.work) cudaFree(B.work);
    B.work_cap = std::max<size_t>(work.size() * 2, 4096);
    OPSB_CUDA(cudaMalloc(&B.work, B.work_cap * sizeof(Work)));
  }
  OPSB_CUDA(cudaMemcpyAsync(B.sys, systems.data(), systems.size() * sizeof(Sys), cudaMemcpyHostToDevice, stream));
  OPSB_CUDA(cudaMemcpyAsync(B.work, work.data(), work.size() * sizeof(Work), cudaMemcpyHostToDevice, stream));
  const int nwork = (int)work.size();
  const int grid = std::min(nwork, 148 * 4);
  if (contig) {
    // 32 chunks per line for n >= 64 (ceil(n/32) rows each), else n/2 chunks of at most 3 rows.
    const int need = std::max(3, (maxn + 31) / 32);
    dim3 blk(32, kLinesContig);
    // (no 4-row variant: with arrays that small the compiler turns the
    // unrolled selects back into indexed accesses and spills them to local memory)
    if (need <= 8) trid_contig_kernel<T, 8><<<grid, blk, 0, stream>>>(B.sys, B.work, nwork);
    else if (need <= 16) trid_contig_kernel<T, 16><<<grid, blk, 0, stream>>>(B.sys, B.work, nwork);
    else throw Error(E_UNSUPPORTED, "tridiagonal lines along x longer than 512 are not supported");
  } else {
    // 16 lines x 16 chunks: a chunk of a 256-point line holds 16 rows, whose
    // four coefficient arrays stay in registers. A chunk holds ceil(n/K) rows
    // for n >= 2K, else at most 3.
    constexpr int L = 16, K = 16;
    const int need = std::max(3, (maxn + K - 1) / K);
    dim3 blk(L, K);
    if (need <= 8) trid_strided_kernel<T, 8, L, K><<<grid, blk, 0, stream>>>(B.sys, B.work, nwork);
    else if (need <= 16) trid_strided_kernel<T, 16, L, K><<<grid, blk, 0, stream>>>(B.sys, B.work, nwork);
    else throw Error(E_UNSUPPORTED, "tridiagonal lines along y/z longer than 256 are not supported");
  }
  OPSB_CUDA(cudaGetLastError());
  if (kernels) (*kernels)++;
}

// Line geometry of a Tridsolver-style strided array: dims (solved extents)
// and pads (allocated extents; element (i,j,k) at i + j*pads[0] + k*pads[0]*pads[1]).
Sys make_sys(const void *a, const void *b, const void *c, void *d, void *u, int ndim, int solvedim, const int *dims,
             const int *pads) {
  if (ndim < 1 || ndim > 3 || solvedim < 0 || solvedim >= ndim) throw Error(E_ARG, "bad ndim/solvedim");
  long long stride[3] = {1, 1, 1};
  for (int k = 1; k < 3; k++) stride[k] = stride[k - 1] * (k - 1 < ndim ? pads[k - 1] : 1);
  Sys s;
  s.a = (const char *)a; s.b = (const char *)b; s.c = (const char *)c;
  s.d = (char *)d; s.u = (char *)u;
  s.n = dims[solvedim];
  s.ss = stride[solvedim];
  int other[2], no = 0;
  for (int k = 0; k < ndim; k++)
    if (k != solvedim) other[no++] = k;
  s.nl0 = no > 0 ? dims[other[0]] : 1;
  s.s0 = no > 0 ? stride[other[0]] : 0;
  s.nl1 = no > 1 ? dims[other[1]] : 1;
  s.s1 = no > 1 ? stride[other[1]] : 0;
  for (int k = 0; k < ndim; k++)
    if (dims[k] < 0 || pads[k] < dims[k]) throw Error(E_ARG, "tridiagonal dims must satisfy 0 <= dims <= pads");
  return s;
}

}  // namespace trid

int capi_guard(const std::function<int()> &f);

// ops_tridMultiDimBatch(_Inc) on dats (ops/c/src/tridiag/ops_tridiag.cpp:78-249).
static int trid_dats(int ndim, int solvedim, const int *range, int a, int b, int c, int d, int u) {
  return capi_guard([&] {
    if (!Runtime::exists()) throw Error(E_STATE, "ops_b200_init has not been called");
    Runtime &r = Runtime::get();
    if (!range) throw Error(E_ARG, "range required");
    Dat &A = r.dat(a), &B = r.dat(b), &C = r.dat(c), &Dd = r.dat(d);
    Dat *U = u >= 0 ? &r.dat(u) : nullptr;
    for (int i = 0; i < 3; i++)
      if (A.size[i] != B.size[i] || B.size[i] != C.size[i] || C.size[i] != Dd.size[i] ||
          (U && U->size[i] != A.size[i]))
        throw Error(E_ARG, "Tridsolver error: the a,b,c,d datasets all need to be the same size");
    if (A.type != B.type || B.type != C.type || C.type != Dd.type || (U && U->type != A.type))
      throw Error(E_ARG, "Tridsolver error: the a,b,c,d datasets must all be of the same type");
    if (A.type != "double" && A.type != "float")
      throw Error(E_UNSUPPORTED, "Tridsolver error: unsupported type. Dataset type must either be \"double\" or \"float\"");
    if (A.pitch != B.pitch || A.pitch != C.pitch || A.pitch != Dd.pitch || (U && U->pitch != A.pitch))
      throw Error(E_ARG, "tridiagonal dats must share one layout");
    r.execute();  // the reference takes raw pointers, which flushes the queue
    int dims[3], pads[3] = {(int)A.pitch, A.size[1], A.size[2]};
    long long offset = 0;
    for (int i = 0; i < ndim; i++) {
      dims[i] = range[2 * i + 1] - range[2 * i];
      if (dims[i] < 0) throw Error(E_ARG, "empty or inverted range");
    }
    offset = range[0] + (ndim > 1 ? (long long)range[2] * A.pitch : 0) + (ndim > 2 ? (long long)range[4] * A.plane : 0);
    const size_t es = A.elem_size;
    auto P = [&](Dat &x) { return x.origin_ptr() + offset * es; };
    std::vector<trid::Sys> sys = {trid::make_sys(P(A), P(B), P(C), P(Dd), U ? P(*U) : nullptr, ndim, solvedim, dims, pads)};
    long long k = 0;
    if (es == 8) trid::launch<double>(sys, solvedim, r.stream(), &k);
    else trid::launch<float>(sys, solvedim, r.stream(), &k);
    r.count_kernels(k);
    return 0;
  });
}

}  // namespace opsb

extern "C" int ops_b200_tridMultiDimBatch(int ndim, int solvedim, const int *range, int a, int b, int c, int d) {
  return opsb::trid_dats(ndim, solvedim, range, a, b, c, d, -1);
}

extern "C" int ops_b200_tridMultiDimBatch_Inc(int ndim, int solvedim, const int *range, int a, int b, int c, int d,
                                              int u) {
  return opsb::trid_dats(ndim, solvedim, range, a, b, c, d, u);
}

extern "C" int ops_b200_trid_batch(int elem_size, int solvedim, int nsys, const ops_b200_trid_system *systems,
                                   void *stream) {
  using namespace opsb;
  return capi_guard([&] {
    if (elem_size != 8 && elem_size != 4) throw Error(E_ARG, "elem_size must be 8 (double) or 4 (float)");
    if (nsys < 0 || (nsys > 0 && !systems)) throw Error(E_ARG, "bad system list");
    std::vector<trid::Sys> sys;
    for (int i = 0; i < nsys; i++) {
      const ops_b200_trid_system &t = systems[i];
      if (!t.a || !t.b || !t.c || !t.d) throw Error(E_ARG, "a, b, c and d are required");
      sys.push_back(trid::make_sys(t.a, t.b, t.c, t.d, t.u, t.ndim, solvedim, t.dims, t.pads));
    }
    long long k = 0;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (elem_size == 8) trid::launch<double>(sys, solvedim, s, &k);
    else trid::launch<float>(sys, solvedim, s, &k);
    if (Runtime::exists()) Runtime::get().count_kernels(k);
    return 0;
  });
}
