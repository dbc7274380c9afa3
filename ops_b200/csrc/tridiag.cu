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
// Every line is split into chunks of about 8 rows, one chunk per thread; a
// thread runs the modified Thomas elimination on its chunk, expressing each
// row through the chunk's first and last unknowns (the partition method of
// Wang 1981, as used for GPUs by Laszlo, Giles and Appleyard, ACM TOMS 42(4)
// 2016):
//   forward, rows 0 and 1 normalised, then for i >= 2
//     r = 1 / (b_i - a_i c'_{i-1}),  d'_i = r (d_i - a_i d'_{i-1}),
//     a'_i = -r a_i a'_{i-1},        c'_i = r c_i;
//   backward for i = m-3 .. 1
//     d'_i -= c'_i d'_{i+1},  a'_i -= c'_i a'_{i+1},  c'_i = -c'_i c'_{i+1};
//   row 0 folds in row 1.
// The chunks' end rows form a small tridiagonal system in shared memory,
// solved by parallel cyclic reduction; a last pass substitutes back. The lines of a work item
// are staged through shared memory, so coefficients and right-hand sides are
// read from HBM once and the solution written once: 40 bytes per FP64
// unknown (48 for _Inc).
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
  long long line0 = 0;  // line kernel: first line number of this system in the launch
  long long scr0 = 0;   // line kernel: first scratch element of this system
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

// One work item = L neighbouring lines x n rows of one system, staged in
// shared memory: the four coefficient tiles are loaded with cp.async (rows
// of the tile along whichever dimension is contiguous in HBM, so the loads
// coalesce), each thread eliminates its chunk of about 8 rows in place in
// shared memory, the chunks' end rows form the reduced system (solved per
// line by Thomas), and the substituted solution is stored with the same
// coalesced mapping. Registers stay few, so two CTAs share an SM and one
// CTA's loads overlap the other's elimination. Tile rows are padded to
// L + 1 elements to spread the chunks over the shared-memory banks.
constexpr int kTileThreads = 256;

#ifndef TRID_CTAS_PER_SM
#define TRID_CTAS_PER_SM 2
#endif
constexpr int kCtasPerSm = TRID_CTAS_PER_SM;
// shared memory per CTA, so that kCtasPerSm CTAs share an SM (227 KB)
constexpr size_t kTileSmem = (size_t)(220 / kCtasPerSm) * 1024;

template <class T>
size_t tile_smem(int L, int n) {
  return (size_t)(4 * (L + 1) * n + 8 * (kTileThreads / L) * L) * sizeof(T);
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
template <class T>
__device__ __forceinline__ void cp_async(T *dst, const T *src) {
  if (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}

template <class T>
__global__ void __launch_bounds__(kTileThreads, kCtasPerSm) trid_tile_kernel(const Sys *__restrict__ sys,
                                                                    const Work *__restrict__ work, int nwork, int L,
                                                                    int nmax) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int P = L + 1;  // padded tile row
  const int tile = P * nmax;
  T *ta = reinterpret_cast<T *>(smraw);
  T *tb = ta + tile, *tc = tb + tile, *td = tc + tile;
  const int K = kTileThreads / L;
  T *RA = td + tile, *RB = RA + 2 * K * L, *RC = RB + 2 * K * L, *RD = RC + 2 * K * L;
  const int tid = threadIdx.x;
  const int l = tid % L, chunk = tid / L;
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const Work wk = work[w];
    const Sys s = sys[wk.sys];
    const int n = s.n;
    const int nl = min(L, s.nl0 - wk.l0);
    const long long base = (long long)wk.l0 * s.s0 + (long long)wk.l1 * s.s1;
    const T *ga = reinterpret_cast<const T *>(s.a) + base;
    const T *gb = reinterpret_cast<const T *>(s.b) + base;
    const T *gc = reinterpret_cast<const T *>(s.c) + base;
    T *gd = reinterpret_cast<T *>(s.d) + base;
    T *gu = s.u ? reinterpret_cast<T *>(s.u) + base : nullptr;
    const bool rows_contig = s.ss == 1;
    const int warp = tid >> 5, lane = tid & 31;
    // 1. stage the four tiles: along x one warp per line (lanes walk the
    // contiguous rows), otherwise thread t takes line t mod L and every
    // (256 / L)-th row from t / L, so each warp-wide copy covers L
    // neighbouring lines of 256 / L rows; no division per element
    if (rows_contig) {
      for (int ll = warp; ll < nl; ll += kTileThreads / 32) {
        const long long g0 = (long long)ll * s.s0;
        for (int i = lane; i < n; i += 32) {
          const int si = i * P + ll;
          cp_async(ta + si, ga + g0 + i);
          cp_async(tb + si, gb + g0 + i);
          cp_async(tc + si, gc + g0 + i);
          cp_async(td + si, gd + g0 + i);
        }
      }
    } else if (l < nl) {
      const long long g0 = (long long)l * s.s0;
      for (int i = chunk; i < n; i += K) {
        const long long g = g0 + (long long)i * s.ss;
        const int si = i * P + l;
        cp_async(ta + si, ga + g);
        cp_async(tb + si, gb + g);
        cp_async(tc + si, gc + g);
        cp_async(td + si, gd + g);
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    // 2. eliminate this thread's chunk in place (same recurrences as chunk_eliminate)
    const int kact = n >= 2 * K ? K : (n / 2 > 0 ? n / 2 : 1);
    const int r0 = chunk * n / kact, r1 = (chunk + 1) * n / kact, m = r1 - r0;
    const bool mine = l < nl && chunk < kact && n > 1;
    if (n == 1 && chunk == 0 && l < nl) td[l] = td[l] * recip(tb[l]);
    if (mine) {
      T pa = T(0), pc = T(0), pd = T(0);
      for (int i = 0; i < m; i++) {
        const int q = (r0 + i) * P + l;
        const T ai = ta[q], bi = tb[q], ci = tc[q], di = td[q];
        T na, nc, nd;
        if (i < 2) {
          const T r = recip(bi);
          na = ai * r;
          nc = ci * r;
          nd = di * r;
        } else {
          const T r = recip(bi - ai * pc);
          nd = r * (di - ai * pd);
          na = -r * ai * pa;
          nc = r * ci;
        }
        ta[q] = na;
        tc[q] = nc;
        td[q] = nd;
        pa = na;
        pc = nc;
        pd = nd;
      }
      const T la = pa, lc = pc, ld = pd;
      if (m > 3) {
        const int q1 = (r0 + m - 2) * P + l;
        T na = ta[q1], nc = tc[q1], nd = td[q1];
        for (int i = m - 3; i >= 1; i--) {
          const int q = (r0 + i) * P + l;
          const T ci = tc[q];
          nd = td[q] - ci * nd;
          na = ta[q] - ci * na;
          nc = -ci * nc;
          ta[q] = na;
          tc[q] = nc;
          td[q] = nd;
        }
      }
      const int q0 = r0 * P + l, q1 = (r0 + 1) * P + l;
      T a0 = ta[q0], c0 = tc[q0], d0 = td[q0];
      if (m > 2) {
        const T r = recip(T(1) - c0 * ta[q1]);
        d0 = r * (d0 - c0 * td[q1]);
        a0 = r * a0;
        c0 = -r * c0 * tc[q1];
        ta[q0] = a0;
        tc[q0] = c0;
        td[q0] = d0;
      }
      RA[(2 * chunk) * L + l] = chunk == 0 ? T(0) : a0;
      RB[(2 * chunk) * L + l] = T(1);
      RC[(2 * chunk) * L + l] = c0;
      RD[(2 * chunk) * L + l] = d0;
      RA[(2 * chunk + 1) * L + l] = la;
      RB[(2 * chunk + 1) * L + l] = T(1);
      RC[(2 * chunk + 1) * L + l] = chunk == kact - 1 ? T(0) : lc;
      RD[(2 * chunk + 1) * L + l] = ld;
    }
    __syncthreads();
    // 3. the reduced system (2 kact rows per line) by parallel cyclic
    // reduction (Hockney 1965): at stride h every row eliminates its
    // neighbours h above and below, log2(2 kact) steps with every chunk
    // thread taking its two rows; afterwards x_k = d_k / b_k.
    if (n > 1) {
      const int N = 2 * kact;
      const bool act = l < nl && chunk < kact;
      for (int h = 1; h < N; h *= 2) {
        T na[2], nb[2], nc[2], nd[2];
        if (act) {
#pragma unroll
          for (int j = 0; j < 2; j++) {
            const int k = 2 * chunk + j;
            const int q = k * L + l;
            T ak = RA[q], bk = RB[q], ck = RC[q], dk = RD[q];
            if (k - h >= 0) {
              const int qm = (k - h) * L + l;
              const T al = -ak * recip(RB[qm]);
              ak = al * RA[qm];
              bk = bk + al * RC[qm];
              dk = dk + al * RD[qm];
            } else {
              ak = T(0);
            }
            if (k + h < N) {
              const int qp = (k + h) * L + l;
              const T ga = -ck * recip(RB[qp]);
              ck = ga * RC[qp];
              bk = bk + ga * RA[qp];
              dk = dk + ga * RD[qp];
            } else {
              ck = T(0);
            }
            na[j] = ak;
            nb[j] = bk;
            nc[j] = ck;
            nd[j] = dk;
          }
        }
        __syncthreads();
        if (act) {
#pragma unroll
          for (int j = 0; j < 2; j++) {
            const int q = (2 * chunk + j) * L + l;
            RA[q] = na[j];
            RB[q] = nb[j];
            RC[q] = nc[j];
            RD[q] = nd[j];
          }
        }
        __syncthreads();
      }
      if (act) {
#pragma unroll
        for (int j = 0; j < 2; j++) {
          const int q = (2 * chunk + j) * L + l;
          RD[q] = RD[q] * recip(RB[q]);
        }
      }
    }
    __syncthreads();
    // 4. substitute back into the d tile
    if (mine) {
      const T xf = RD[(2 * chunk) * L + l], xl = RD[(2 * chunk + 1) * L + l];
      for (int i = 0; i < m; i++) {
        const int q = (r0 + i) * P + l;
        td[q] = (i == 0) ? xf : (i == m - 1) ? xl : td[q] - ta[q] * xf - tc[q] * xl;
      }
    }
    __syncthreads();
    // 5. store (d = x, or u += x), with the loads' mapping
    if (rows_contig) {
      for (int ll = warp; ll < nl; ll += kTileThreads / 32) {
        const long long g0 = (long long)ll * s.s0;
        for (int i = lane; i < n; i += 32) {
          const T x = td[i * P + ll];
          if (gu) gu[g0 + i] += x;
          else gd[g0 + i] = x;
        }
      }
    } else if (l < nl) {
      const long long g0 = (long long)l * s.s0;
      for (int i = chunk; i < n; i += K) {
        const long long g = g0 + (long long)i * s.ss;
        const T x = td[i * P + l];
        if (gu) gu[g] += x;
        else gd[g] = x;
      }
    }
    __syncthreads();
  }
}

// x sweeps (lines contiguous in HBM) of up to 32 R rows, no block-wide
// barriers: a warp solves 32 / P lines at once, P lanes per line (P = 32,
// 16 or 8: the fewest lanes whose chunks of at most R rows cover a line, so
// short lines share a warp). The warp stages its lines' a, b, c, d through
// its own strip of shared memory with coalesced cp.async copies (row r at
// r + r / 8, so that lanes reading neighbouring chunks hit different
// banks), every lane eliminates its chunk in registers by the same partition
// recurrences as trid_tile_kernel, each line's 2 P chunk end rows are solved
// by parallel cyclic reduction over shuffles within its lane group, and the
// lanes substitute back and store through the strip. A warp keeps all its
// lines' 4 n loads in flight at once.
constexpr int kWarpLines = 8;  // warps per CTA

template <int R>
__host__ __device__ constexpr int warp_strip(int) { return 32 * R + 4 * R + 2; }
__device__ __forceinline__ int strip_pos(int r) { return r + (r >> 3); }
// Lanes per line for lines of n rows and chunks of at most R rows.
__host__ __device__ inline int lanes_per_line(int n, int R) {
  int p = 32;
  while (p > 8 && (p / 2) * R >= n) p /= 2;
  return p;
}

// FP32 lines hold half the registers: three CTAs per SM. FP: lanes per
// line fixed at compile time (32: every line of the launch fills a warp), or
// 0 to choose per system.
template <class T, int R, int FP>
__global__ void __launch_bounds__(32 * kWarpLines, sizeof(T) == 4 ? 3 : 2)
    trid_warp_kernel(const Sys *__restrict__ sys, const Work *__restrict__ work, int nwork) {
  extern __shared__ __align__(16) unsigned char smraw[];
  constexpr int SW = warp_strip<R>(0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T *Sa = reinterpret_cast<T *>(smraw) + (size_t)warp * 4 * SW;
  T *Sb = Sa + SW, *Sc = Sb + SW, *Sd = Sc + SW;
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const Work wk = work[w];
    const Sys s = sys[wk.sys];
    const int n = s.n;
    const int P = FP ? FP : lanes_per_line(n, R), G = 32 / P;  // lanes per line, lines per warp
    const int line0 = wk.l0 + warp * G;               // this warp's first line
    if (line0 >= s.nl0) continue;                     // the same for the whole warp
    const long long base0 = (long long)line0 * s.s0 + (long long)wk.l1 * s.s1;
    const T *ga = reinterpret_cast<const T *>(s.a) + base0;
    const T *gb = reinterpret_cast<const T *>(s.b) + base0;
    const T *gc = reinterpret_cast<const T *>(s.c) + base0;
    T *gd = reinterpret_cast<T *>(s.d) + base0;
    T *gu = s.u ? reinterpret_cast<T *>(s.u) + base0 : nullptr;
    const int nlines = min(G, s.nl0 - line0);
    // asynchronous copies, line by line over the whole warp: every load in flight at once
    for (int g = 0; g < nlines; g++) {
      const long long lo = (long long)g * s.s0;
      const int ro = g * P * R;
      for (int i = lane; i < n; i += 32) {
        const int p = strip_pos(ro + i);
        cp_async(Sa + p, ga + lo + i);
        cp_async(Sb + p, gb + lo + i);
        cp_async(Sc + p, gc + lo + i);
        cp_async(Sd + p, gd + lo + i);
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncwarp();
    // 1. this lane's chunk of its line: forward and backward partition sweeps in registers
    const int g = lane / P, gl = lane - g * P, ro = g * P * R;
    const int kact = n >= 2 * P ? P : (n / 2 > 0 ? n / 2 : 1);
    const int r0 = ro + gl * n / kact, m = (gl + 1) * n / kact - gl * n / kact;
    const bool act = g < nlines && gl < kact && n > 1;
    T ra[R], rc[R], rd[R];
    T fa[2] = {T(0), T(0)}, fb[2] = {T(1), T(1)}, fc[2] = {T(0), T(0)}, fd[2] = {T(0), T(0)};
    if (act) {
      T pa = T(0), pc = T(0), pd = T(0);
#pragma unroll
      for (int i = 0; i < R; i++) {
        if (i < m) {
          const int p = strip_pos(r0 + i);
          const T ai = Sa[p], bi = Sb[p], ci = Sc[p], di = Sd[p];
          T na, nc, nd;
          if (i < 2) {
            const T r = recip(bi);
            na = ai * r;
            nc = ci * r;
            nd = di * r;
          } else {
            const T r = recip(bi - ai * pc);
            nd = r * (di - ai * pd);
            na = -r * ai * pa;
            nc = r * ci;
          }
          ra[i] = na;
          rc[i] = nc;
          rd[i] = nd;
          pa = na;
          pc = nc;
          pd = nd;
        }
      }
      fa[1] = pa;
      fc[1] = gl == kact - 1 ? T(0) : pc;
      fd[1] = pd;
      // backward: rows m-3 .. 1 fold in row i + 1 (whose values ride in
      // na, nc, nd; rows from m-2 up pass theirs on unchanged)
      T na = T(0), nc = T(0), nd = T(0);
#pragma unroll
      for (int t = 0; t < R - 1; t++) {
        const int i = R - 1 - t;
        if (i <= m - 3) {
          const T ci = rc[i];
          nd = rd[i] - ci * nd;
          na = ra[i] - ci * na;
          nc = -ci * nc;
          ra[i] = na;
          rc[i] = nc;
          rd[i] = nd;
        } else {
          na = ra[i];
          nc = rc[i];
          nd = rd[i];
        }
      }
      T a0 = ra[0], c0 = rc[0], d0 = rd[0];
      if (m > 2) {
        const T r = recip(T(1) - c0 * ra[1]);
        d0 = r * (d0 - c0 * rd[1]);
        a0 = r * a0;
        c0 = -r * c0 * rc[1];
      }
      ra[0] = a0;
      rc[0] = c0;
      rd[0] = d0;
      fa[0] = gl == 0 ? T(0) : a0;
      fc[0] = c0;
      fd[0] = d0;
    }
    // 2. each line's 2 P chunk end rows (row 2 gl + j), parallel cyclic
    // reduction over shuffles within the line's lane group; lanes without a
    // chunk hold identity rows
    const int N = 2 * P;
    for (int h = 1; h < N; h *= 2) {
      T ma[2], mb[2], mc[2], md[2], pa[2], pb[2], pc[2], pd[2];
      if (h == 1) {
        ma[0] = __shfl_up_sync(0xffffffffu, fa[1], 1, P);
        mb[0] = __shfl_up_sync(0xffffffffu, fb[1], 1, P);
        mc[0] = __shfl_up_sync(0xffffffffu, fc[1], 1, P);
        md[0] = __shfl_up_sync(0xffffffffu, fd[1], 1, P);
        pa[1] = __shfl_down_sync(0xffffffffu, fa[0], 1, P);
        pb[1] = __shfl_down_sync(0xffffffffu, fb[0], 1, P);
        pc[1] = __shfl_down_sync(0xffffffffu, fc[0], 1, P);
        pd[1] = __shfl_down_sync(0xffffffffu, fd[0], 1, P);
        pa[0] = fa[1]; pb[0] = fb[1]; pc[0] = fc[1]; pd[0] = fd[1];
        ma[1] = fa[0]; mb[1] = fb[0]; mc[1] = fc[0]; md[1] = fd[0];
      } else {
        const int q = h >> 1;
#pragma unroll
        for (int j = 0; j < 2; j++) {
          ma[j] = __shfl_up_sync(0xffffffffu, fa[j], q, P);
          mb[j] = __shfl_up_sync(0xffffffffu, fb[j], q, P);
          mc[j] = __shfl_up_sync(0xffffffffu, fc[j], q, P);
          md[j] = __shfl_up_sync(0xffffffffu, fd[j], q, P);
          pa[j] = __shfl_down_sync(0xffffffffu, fa[j], q, P);
          pb[j] = __shfl_down_sync(0xffffffffu, fb[j], q, P);
          pc[j] = __shfl_down_sync(0xffffffffu, fc[j], q, P);
          pd[j] = __shfl_down_sync(0xffffffffu, fd[j], q, P);
        }
      }
#pragma unroll
      for (int j = 0; j < 2; j++) {
        const int k = 2 * gl + j;
        T ak = fa[j], bk = fb[j], ck = fc[j], dk = fd[j];
        if (k - h >= 0) {
          const T al = -ak * recip(mb[j]);
          ak = al * ma[j];
          bk = bk + al * mc[j];
          dk = dk + al * md[j];
        } else {
          ak = T(0);
        }
        if (k + h < N) {
          const T gg = -ck * recip(pb[j]);
          ck = gg * pc[j];
          bk = bk + gg * pa[j];
          dk = dk + gg * pd[j];
        } else {
          ck = T(0);
        }
        fa[j] = ak;
        fb[j] = bk;
        fc[j] = ck;
        fd[j] = dk;
      }
    }
    // 3. substitute back, then store through the strip with the loads' mapping
    if (act) {
      const T xf = fd[0] * recip(fb[0]), xl = fd[1] * recip(fb[1]);
#pragma unroll
      for (int i = 0; i < R; i++)
        if (i < m) Sd[strip_pos(r0 + i)] = (i == 0) ? xf : (i == m - 1) ? xl : rd[i] - ra[i] * xf - rc[i] * xl;
    }
    if (n == 1 && gl == 0 && g < nlines) Sd[strip_pos(ro)] = Sd[strip_pos(ro)] * recip(Sb[strip_pos(ro)]);
    __syncwarp();
    for (int gg = 0; gg < nlines; gg++) {
      const long long lo = (long long)gg * s.s0;
      const int rg = gg * P * R;
      for (int i = lane; i < n; i += 32) {
        const T x = Sd[strip_pos(rg + i)];
        if (gu) gu[lo + i] += x;
        else gd[lo + i] = x;
      }
    }
    __syncwarp();
  }
}

// Lines strided along the solve dimension and contiguous across lines (the
// y and z sweeps): one thread per line runs the Thomas algorithm straight
// from HBM, neighbouring threads reading neighbouring lines so every access
// coalesces. The forward pass keeps c' and d' in a scratch array laid out
// row-major over the system's lines (coalesced too) and the backward pass
// reads them back: 72 bytes per FP64 unknown (80 for _Inc) against the
// tile kernel's 40, but no staging, no barriers and several rows of loads in
// flight per thread, which is what the strided sweeps lacked. Rows in
// flight: 8 (one 32-byte sector of each line per array in FP32, two in
// FP64), or 4 in FP64 when the lines fill the GPU (more than 1024 a SM): a
// grid of few lines leaves the registers free and gains from the deeper
// pipeline (256^3 FP64 y sweep 0.239 -> 0.219 ms), while the 64-block batch
// (about 0.5 M lines) lost 7-20 % with it. The arithmetic is the textbook
// Thomas elimination:
//   c'_0 = c_0 / b_0, d'_0 = d_0 / b_0; for i >= 1, r = 1 / (b_i - a_i c'_{i-1}),
//   c'_i = c_i r, d'_i = (d_i - a_i d'_{i-1}) r; x_{n-1} = d'_{n-1},
//   x_i = d'_i - c'_i x_{i+1}.
constexpr int kLineThreads = 128;
constexpr long long kLinesDeep = 148LL * 1024;  // at most this many lines: 8 rows in flight in FP64

template <class T, int kLineUnroll>
__global__ void __launch_bounds__(kLineThreads) trid_line_kernel(const Sys *__restrict__ sys, int nsys,
                                                                 long long total, T *__restrict__ scr_c,
                                                                 T *__restrict__ scr_d) {
  for (long long g = (long long)blockIdx.x * kLineThreads + threadIdx.x; g < total;
       g += (long long)gridDim.x * kLineThreads) {
    int lo = 0, hi = nsys - 1;  // last system whose first line is <= g
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (sys[mid].line0 <= g) lo = mid;
      else hi = mid - 1;
    }
    const Sys &s = sys[lo];
    const long long k = g - s.line0, nlines = (long long)s.nl0 * s.nl1;
    const int n = s.n;
    const long long base = (k % s.nl0) * s.s0 + (k / s.nl0) * s.s1, ss = s.ss;
    const T *a = reinterpret_cast<const T *>(s.a) + base;
    const T *b = reinterpret_cast<const T *>(s.b) + base;
    const T *c = reinterpret_cast<const T *>(s.c) + base;
    const T *d = reinterpret_cast<const T *>(s.d) + base;
    T *x = reinterpret_cast<T *>(s.d) + base;
    T *u = s.u ? reinterpret_cast<T *>(s.u) + base : nullptr;
    T *cp = scr_c + s.scr0 + k, *dp = scr_d + s.scr0 + k;
    if (n <= 0) continue;
    T r = recip(b[0]);
    T pc = c[0] * r, pd = d[0] * r;
    cp[0] = pc;
    dp[0] = pd;
    int i = 1;
    for (; i + kLineUnroll <= n; i += kLineUnroll) {
      T ai[kLineUnroll], bi[kLineUnroll], ci[kLineUnroll], di[kLineUnroll];
#pragma unroll
      for (int j = 0; j < kLineUnroll; j++) {
        const long long q = (long long)(i + j) * ss;
        ai[j] = a[q];
        bi[j] = b[q];
        ci[j] = c[q];
        di[j] = d[q];
      }
#pragma unroll
      for (int j = 0; j < kLineUnroll; j++) {
        r = recip(bi[j] - ai[j] * pc);
        pc = ci[j] * r;
        pd = (di[j] - ai[j] * pd) * r;
        cp[(long long)(i + j) * nlines] = pc;
        dp[(long long)(i + j) * nlines] = pd;
      }
    }
    for (; i < n; i++) {
      const long long q = (long long)i * ss;
      const T ai = a[q];
      r = recip(b[q] - ai * pc);
      pc = c[q] * r;
      pd = (d[q] - ai * pd) * r;
      cp[(long long)i * nlines] = pc;
      dp[(long long)i * nlines] = pd;
    }
    T xv = pd;  // x_{n-1}
    {
      const long long q = (long long)(n - 1) * ss;
      if (u) u[q] += xv;
      else x[q] = xv;
    }
    int j = n - 2;
    for (; j - kLineUnroll + 1 >= 0; j -= kLineUnroll) {
      T cj[kLineUnroll], dj[kLineUnroll];
#pragma unroll
      for (int t = 0; t < kLineUnroll; t++) {
        cj[t] = cp[(long long)(j - t) * nlines];
        dj[t] = dp[(long long)(j - t) * nlines];
      }
#pragma unroll
      for (int t = 0; t < kLineUnroll; t++) {
        xv = dj[t] - cj[t] * xv;
        const long long q = (long long)(j - t) * ss;
        if (u) u[q] += xv;
        else x[q] = xv;
      }
    }
    for (; j >= 0; j--) {
      xv = dp[(long long)j * nlines] - cp[(long long)j * nlines] * xv;
      const long long q = (long long)j * ss;
      if (u) u[q] += xv;
      else x[q] = xv;
    }
  }
}

// Device copies of the work description, grown as needed.
struct Buffers {
  Sys *sys = nullptr;
  Work *work = nullptr;
  size_t sys_cap = 0, work_cap = 0;
  void *scr = nullptr;  // line kernel scratch (c' then d')
  size_t scr_bytes = 0;
};
Buffers &buffers() {
  static Buffers b;
  return b;
}

// The y/z sweeps (solve dimension strided, lines contiguous) by the line
// kernel; returns false when some system does not have that shape (the x
// sweeps stay with the tile kernel: a warp-transposing variant of the line
// kernel for them measured 0.70 ms against the tile kernel's 0.41 ms on the
// 256^3 FP64 x sweep).
template <class T>
bool launch_lines(std::vector<Sys> systems, cudaStream_t stream, long long *kernels) {
  long long lines = 0, unknowns = 0;
  for (Sys &s : systems) {
    if (s.ss == 1 || s.s0 != 1) return false;
    s.line0 = lines;
    s.scr0 = unknowns;
    const long long nl = (long long)s.nl0 * s.nl1;
    lines += s.n > 0 ? nl : 0;
    unknowns += s.n > 0 ? nl * s.n : 0;
  }
  std::vector<Sys> live;  // systems with no rows or no lines take no part

  for (const Sys &s : systems)
    if (s.n > 0 && (long long)s.nl0 * s.nl1 > 0) live.push_back(s);
  if (live.empty()) return true;
  Buffers &B = buffers();
  if (B.sys_cap < live.size()) {
    if (B.sys) cudaFree(B.sys);
    B.sys_cap = std::max<size_t>(live.size(), 64);
    OPSB_CUDA(cudaMalloc(&B.sys, B.sys_cap * sizeof(Sys)));
  }
  const size_t need = 2 * (size_t)unknowns * sizeof(T);
  if (B.scr_bytes < need) {
    if (B.scr) cudaFree(B.scr);
    B.scr = nullptr;
    OPSB_CUDA(cudaMalloc(&B.scr, need));
    B.scr_bytes = need;
  }
  OPSB_CUDA(cudaMemcpyAsync(B.sys, live.data(), live.size() * sizeof(Sys), cudaMemcpyHostToDevice, stream));
  T *sc = static_cast<T *>(B.scr), *sd = sc + unknowns;
  const int grid = (int)std::min<long long>((lines + kLineThreads - 1) / kLineThreads, 148LL * 16);
  if (sizeof(T) == 4 || lines <= kLinesDeep)
    trid_line_kernel<T, 8><<<grid, kLineThreads, 0, stream>>>(B.sys, (int)live.size(), lines, sc, sd);
  else
    trid_line_kernel<T, 4><<<grid, kLineThreads, 0, stream>>>(B.sys, (int)live.size(), lines, sc, sd);
  OPSB_CUDA(cudaGetLastError());
  if (kernels) (*kernels)++;
  return true;
}

// "trid_warp" option: -1 and 1 use the warp kernel whenever it applies, 0 never.
int &warp_mode() {
  static int m = -1;
  return m;
}
void set_warp_mode(int m) {
  if (m < -1 || m > 1) throw Error(E_ARG, "trid_warp must be -1, 0 or 1");
  warp_mode() = m;
}

template <class T, int R, int FP>
void launch_warp(const Buffers &B, int nwork, cudaStream_t stream) {
  const int smem = (int)(kWarpLines * 4 * warp_strip<R>(0) * sizeof(T));
  static int occupancy = 0;  // CTAs per SM, per instantiation
  if (occupancy == 0) {
    OPSB_CUDA(cudaFuncSetAttribute(trid_warp_kernel<T, R, FP>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    OPSB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occupancy, trid_warp_kernel<T, R, FP>,
                                                            32 * kWarpLines, smem));
    occupancy = std::max(occupancy, 1);
  }
  const int grid = std::min(nwork, 148 * occupancy);
  trid_warp_kernel<T, R, FP><<<grid, 32 * kWarpLines, smem, stream>>>(B.sys, B.work, nwork);
  OPSB_CUDA(cudaGetLastError());
}

template <class T>
void launch(const std::vector<Sys> &systems, int solvedim, cudaStream_t stream, long long *kernels) {
  (void)solvedim;
  int maxn = 0;
  for (const Sys &s : systems) maxn = std::max(maxn, s.n);
  if (maxn == 0) return;
  if (launch_lines<T>(systems, stream, kernels)) return;
  bool contig = true;
  for (const Sys &s : systems) contig = contig && (s.n == 0 || s.ss == 1);
  // x sweeps of lines up to 256 rows: a warp per 1, 2 or 4 lines
  // (trid_warp_kernel); longer lines, or the option set to 0, take the tile
  // kernel
  const int wm = warp_mode();
  const bool warp_path = contig && maxn <= 256 && wm != 0;
  const int wR = maxn <= 128 ? 4 : 8;  // rows per lane of the warp kernel
  // tile kernel: lines per work item, the largest power of two (<= 64) whose tiles fit
  int L = 64;
  if (!warp_path) {
    while (L > 1 && tile_smem<T>(L, maxn) > kTileSmem) L /= 2;
    if (tile_smem<T>(L, maxn) > kTileSmem) throw Error(E_UNSUPPORTED, "tridiagonal lines longer than the tile budget");
  }
  std::vector<Work> work;
  for (int i = 0; i < (int)systems.size(); i++) {
    const Sys &s = systems[i];
    if (s.n == 0) continue;
    // warp kernel: a CTA's warps take kWarpLines x (lines per warp) lines
    const int Ls = warp_path ? kWarpLines * (32 / lanes_per_line(s.n, wR)) : L;
    for (int l1 = 0; l1 < s.nl1; l1++)
      for (int l0 = 0; l0 < s.nl0; l0 += Ls) work.push_back({i, l0, l1});
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
  if (warp_path) {
    bool full = true;  // every line needs all 32 lanes
    for (const Sys &s : systems) full = full && (s.n == 0 || lanes_per_line(s.n, wR) == 32);
    if (wR == 4)
      full ? launch_warp<T, 4, 32>(B, nwork, stream) : launch_warp<T, 4, 0>(B, nwork, stream);
    else
      full ? launch_warp<T, 8, 32>(B, nwork, stream) : launch_warp<T, 8, 0>(B, nwork, stream);
    if (kernels) (*kernels)++;
    return;
  }
  const size_t smem = tile_smem<T>(L, maxn);
  static size_t attr_set = 0;
  if (smem > attr_set) {
    OPSB_CUDA(cudaFuncSetAttribute(trid_tile_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_set = smem;
  }
  const int per_sm = std::max(1, std::min(kCtasPerSm, (int)(233472 / (smem + 1024))));
  const int grid = std::min(nwork, 148 * per_sm);
  trid_tile_kernel<T><<<grid, kTileThreads, smem, stream>>>(B.sys, B.work, nwork, L, maxn);
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
    // a line solve needs its whole line on one GPU: no partitioned dats
    if (A.split >= 0 || B.split >= 0 || C.split >= 0 || Dd.split >= 0 || (U && U->split >= 0))
      throw Error(E_UNSUPPORTED, "Tridsolver: dats partitioned across ranks are not supported");
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
