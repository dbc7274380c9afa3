// tcgen05 implicit-GEMM 3x3 convolution; design notes in conv_tc.cuh.
#include <cuda.h>

#include <cstdio>
#include <cstring>

#include "conv_tc.cuh"

namespace opsb {
namespace cnn {
namespace {

constexpr int kTileM = 128;
constexpr int kThreads = 192;
constexpr unsigned long long kWaitNs = 2000000000ull;  // a stuck mbarrier wait gives up after 2 s

enum { ERR_NONE = 0, ERR_WAIT_WEIGHTS = 1, ERR_WAIT_EMPTY = 2, ERR_WAIT_FULL = 3, ERR_WAIT_ACC_EMPTY = 4,
       ERR_WAIT_ACC_FULL = 5 };

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait on one phase; false when it expired or another role aborted.
__device__ __noinline__ bool mbar_wait(uint64_t *b, unsigned parity, volatile int *abort_flag) {
  const unsigned long long t0 = now_ns();
  for (unsigned i = 0;; i++) {
    if (mbar_try(b, parity)) return true;
    if ((i & 255u) == 255u) {
      if (*abort_flag) return false;
      if (now_ns() - t0 > kWaitNs) return false;
    }
  }
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1, int c2,
                                            int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], "
      "[%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];" ::
          "r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

// Shared-memory matrix descriptor (tcgen05): start address, leading byte
// offset 16 (unused by swizzled K-major layouts), stride byte offset between
// 8-row groups, descriptor version 1, swizzle layout type.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t sbo_bytes, uint32_t layout) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;
  d |= (uint64_t)(layout & 7u) << 61;
  return d;
}

// Instruction descriptor, kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t instr_desc(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  const uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(mask0), "r"(mask1), "r"(mask2), "r"(mask3));
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ void record_error(int *err, volatile int *abort_flag, int code) {
  atomicCAS(err, 0, code);
  *abort_flag = 1;
}

template <int CIN, int COUT>
struct Cfg {
  static constexpr int S = CIN * 2;                    // bytes per pixel row = swizzle span
  static constexpr uint32_t LAYOUT = CIN == 16 ? 6u : CIN == 32 ? 4u : 2u;  // SW32 / SW64 / SW128
  // 128-pixel MMA blocks per tile: at 16 input channels one TMA box per tap
  // carries 4 blocks (16 KB instead of 4 KB; 4096^2 16->16 826 -> 665 us);
  // at 32 channels 2 blocks a box measured slower (358 -> 407 us at 2048^2
  // 32->32), at 64 no change, so those keep one block a box
  static constexpr int SUB = CIN == 16 ? 4 : 1;
  static constexpr int A_BYTES = SUB * kTileM * S;
  static constexpr int W_TAP = COUT * S;
  static constexpr int W_BYTES = 9 * W_TAP;
  static constexpr int STAGES = SUB > 1 ? 6 : 8;
  static constexpr int NACC = SUB > 1 ? 2 : 4;         // accumulator sets in tensor memory
  static constexpr int TMEM_COLS = NACC * SUB * COUT;  // 64, 128 or 256 columns
  static constexpr int OFF_W = 0;
  static constexpr int OFF_A = (W_BYTES + 1023) / 1024 * 1024;
  static constexpr int OFF_BAR = OFF_A + STAGES * A_BYTES;
  static constexpr int NBAR = 2 * STAGES + 2 * NACC + 1;
  static constexpr int SMEM = OFF_BAR + NBAR * 8 + 16 + 1024;  // + alignment slack
  static_assert(COUT % 16 == 0 && COUT >= 16 && COUT <= 64, "Cout");
  static_assert(CIN == 16 || CIN == 32 || CIN == 64, "Cin");
  static_assert(TMEM_COLS >= 32 && (TMEM_COLS & (TMEM_COLS - 1)) == 0, "tmem columns");
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(kThreads, 1)
    conv3x3_tc_kernel(const __grid_constant__ CUtensorMap xmap, const __grid_constant__ CUtensorMap wmap,
                      ConvArgs a) {
  using C = Cfg<CIN, COUT>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  uint8_t *sW = smem + C::OFF_W;
  uint8_t *sA = smem + C::OFF_A;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + C::OFF_BAR);
  uint64_t *full = bars, *empty = bars + C::STAGES, *acc_full = bars + 2 * C::STAGES,
           *acc_empty = acc_full + C::NACC, *wbar = acc_empty + C::NACC;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + C::NBAR);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < C::STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < C::NACC; b++) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 4);
    }
    mbar_init(wbar, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"((uint32_t)C::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int per_img = a.tiles_x * a.tiles_y;

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      uint32_t pending = 0;              // stages with a load in flight
      uint32_t pend_par = 0;             // their phase parity
      mbar_expect_tx(wbar, C::W_BYTES);
      tma_load_3d(sW, &wmap, wbar, 0, 0, 0);
      int s = 0;
      uint32_t ph = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < a.tiles && ok; t += gridDim.x) {
        const int img = t / per_img, rem = t - img * per_img;
        const int ty = rem / a.tiles_x, tx = rem - ty * a.tiles_x;
        const int w0 = tx * a.tw, h0 = ty * a.th;
        for (int tap = 0; tap < 9; tap++) {
          if (!mbar_wait(&empty[s], ph ^ 1u, abort_flag)) {
            record_error(a.err, abort_flag, ERR_WAIT_EMPTY);
            ok = false;
            break;
          }
          pending &= ~(1u << s);  // the MMAs that read the previous load of this stage are done
          mbar_expect_tx(&full[s], C::A_BYTES);
          tma_load_4d(sA + s * C::A_BYTES, &xmap, &full[s], 0, w0 + tap % 3 - 1, h0 + tap / 3 - 1, img);
          pending |= 1u << s;
          pend_par = (pend_par & ~(1u << s)) | (ph << s);
          if (++s == C::STAGES) {
            s = 0;
            ph ^= 1u;
          }
        }
      }
      if (!ok) {
        // let the copies already issued land before the CTA exits (bounded)
        volatile int never = 0;
        for (int k = 0; k < C::STAGES; k++)
          if (pending & (1u << k)) mbar_wait(&full[k], (pend_par >> k) & 1u, &never);
        mbar_wait(wbar, 0, &never);
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer (one thread) ----------------
    if (lane == 0) {
      constexpr uint32_t IDESC = instr_desc(kTileM, COUT);
      const uint32_t sA0 = smem_u32(sA), sW0 = smem_u32(sW);
      bool ok = mbar_wait(wbar, 0, abort_flag);
      if (!ok) record_error(a.err, abort_flag, ERR_WAIT_WEIGHTS);
      int s = 0, b = 0;
      uint32_t ph = 0, aph = 0;
      bool issued = false;
      uint64_t *last_commit = nullptr;
      uint32_t last_par = 0;
      for (int t = blockIdx.x; t < a.tiles && ok; t += gridDim.x) {
        if (!mbar_wait(&acc_empty[b], aph ^ 1u, abort_flag)) {
          record_error(a.err, abort_flag, ERR_WAIT_ACC_EMPTY);
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(b * C::SUB * COUT);
        for (int tap = 0; tap < 9 && ok; tap++) {
          if (!mbar_wait(&full[s], ph, abort_flag)) {
            record_error(a.err, abort_flag, ERR_WAIT_FULL);
            ok = false;
            break;
          }
          tc_fence_after();
#pragma unroll
          for (int j = 0; j < C::SUB; j++)
#pragma unroll
            for (int kb = 0; kb < CIN / 16; kb++) {
              const uint64_t ad =
                  smem_desc(sA0 + s * C::A_BYTES + j * kTileM * C::S + kb * 32, 8 * C::S, C::LAYOUT);
              const uint64_t bd = smem_desc(sW0 + tap * C::W_TAP + kb * 32, 8 * C::S, C::LAYOUT);
              umma_bf16(d + (uint32_t)(j * COUT), ad, bd, IDESC, (tap | kb) != 0 ? 1u : 0u);
            }
          umma_commit(&empty[s]);
          issued = true;
          last_commit = &empty[s];
          last_par = ph;
          if (++s == C::STAGES) {
            s = 0;
            ph ^= 1u;
          }
        }
        if (!ok) break;
        umma_commit(&acc_full[b]);
        if (++b == C::NACC) {
          b = 0;
          aph ^= 1u;
        }
      }
      if (!ok && issued) {
        // MMAs complete in order: the last commit's phase covers all of them (bounded)
        volatile int never = 0;
        mbar_wait(last_commit, last_par, &never);
      }
    }
  } else {
    // ---------------- epilogue: warps 2..5 ----------------
    const int q = warp & 3;
    const int row = q * 32 + lane;
    int b = 0;
    uint32_t aph = 0;
    for (int t = blockIdx.x; t < a.tiles; t += gridDim.x) {
      int ok = 1;
      if (lane == 0) {
        ok = mbar_wait(&acc_full[b], aph, abort_flag) ? 1 : 0;
        if (!ok) record_error(a.err, abort_flag, ERR_WAIT_ACC_FULL);
      }
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) break;
      tc_fence_after();
      const int img = t / per_img, rem = t - img * per_img;
      const int ty = rem / a.tiles_x, tx = rem - ty * a.tiles_x;
#pragma unroll 1
      for (int j = 0; j < C::SUB; j++) {
        float v[COUT];
        const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)((b * C::SUB + j) * COUT);
#pragma unroll
        for (int c = 0; c < COUT; c += 16) tmem_ld16(taddr + c, v + c);
        tmem_wait_ld();
        if (j == C::SUB - 1) {  // this accumulator set is read: the MMA warp may reuse it
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&acc_empty[b]);
        }
        const int p = j * kTileM + row;  // pixel of the tile (row-major over tw x th)
        const int x = tx * a.tw + p % a.tw, y = ty * a.th + p / a.tw;
        if (x >= a.w || y >= a.h) continue;
        const size_t pix = ((size_t)img * a.h + y) * a.w + x;
        if (a.mode == CONV_BIAS_RELU || a.mode == CONV_BIAS) {
#pragma unroll
          for (int c = 0; c < COUT; c++) {
            float o = v[c] + a.bias[c];
            v[c] = (a.mode == CONV_BIAS_RELU) ? fmaxf(o, 0.0f) : o;
          }
        } else if (a.mode == CONV_MASK) {
          const uint4 *mp = reinterpret_cast<const uint4 *>(a.mask + pix * COUT);
#pragma unroll
          for (int c8 = 0; c8 < COUT / 8; c8++) {
            uint4 m = mp[c8];
            const __nv_bfloat16 *mb = reinterpret_cast<const __nv_bfloat16 *>(&m);
#pragma unroll
            for (int k = 0; k < 8; k++)
              if (!(__bfloat162float(mb[k]) > 0.0f)) v[c8 * 8 + k] = 0.0f;
          }
        }
        uint4 *yp = reinterpret_cast<uint4 *>(a.y + pix * COUT);
#pragma unroll
        for (int c8 = 0; c8 < COUT / 8; c8++) {
          uint4 o;
          __nv_bfloat162 *ob = reinterpret_cast<__nv_bfloat162 *>(&o);
#pragma unroll
          for (int k = 0; k < 4; k++) ob[k] = __floats2bfloat162_rn(v[c8 * 8 + 2 * k], v[c8 * 8 + 2 * k + 1]);
          yp[c8] = o;
        }
      }
      if (++b == C::NACC) {
        b = 0;
        aph ^= 1u;
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)C::TMEM_COLS));
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// The driver's tensor-map encoder, resolved through the runtime so that the
// library does not link libcuda directly.
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encoder() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

bool encode(CUtensorMap *m, int rank, const void *base, const cuuint64_t *dims, const cuuint64_t *strides,
            const cuuint32_t *box, CUtensorMapSwizzle sw) {
  EncodeTiledFn fn = encoder();
  if (!fn) return false;
  cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, (cuuint32_t)rank, const_cast<void *>(base), dims, strides, box,
                  estr, CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <int CIN, int COUT>
cudaError_t launch(const __nv_bfloat16 *x, const __nv_bfloat16 *w, const ConvArgs &args, cudaStream_t s) {
  using C = Cfg<CIN, COUT>;
  const CUtensorMapSwizzle sw = CIN == 16 ? CU_TENSOR_MAP_SWIZZLE_32B
                                          : CIN == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B;
  CUtensorMap xm, wm;
  cuuint64_t xd[4] = {(cuuint64_t)CIN, (cuuint64_t)args.w, (cuuint64_t)args.h, (cuuint64_t)args.n};
  cuuint64_t xs[3] = {(cuuint64_t)CIN * 2, (cuuint64_t)args.w * CIN * 2, (cuuint64_t)args.h * args.w * CIN * 2};
  cuuint32_t xb[4] = {(cuuint32_t)CIN, (cuuint32_t)args.tw, (cuuint32_t)args.th, 1};
  if (!encode(&xm, 4, x, xd, xs, xb, sw)) return cudaErrorInvalidValue;
  cuuint64_t wd[3] = {(cuuint64_t)CIN, (cuuint64_t)COUT, 9};
  cuuint64_t ws[2] = {(cuuint64_t)CIN * 2, (cuuint64_t)COUT * CIN * 2};
  cuuint32_t wb[3] = {(cuuint32_t)CIN, (cuuint32_t)COUT, 9};
  if (!encode(&wm, 3, w, wd, ws, wb, sw)) return cudaErrorInvalidValue;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(conv3x3_tc_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         C::SMEM);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  // resident CTAs per SM: shared memory (228 KB, 1 KB reserved per CTA) and
  // tensor memory (512 columns) both bound it
  int per_sm = 233472 / (C::SMEM + 1024);
  if (per_sm > 512 / C::TMEM_COLS) per_sm = 512 / C::TMEM_COLS;
  if (per_sm > 4) per_sm = 4;
  if (per_sm < 1) per_sm = 1;
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int grid = sms * per_sm;
  if (grid > args.tiles) grid = args.tiles;
  conv3x3_tc_kernel<CIN, COUT><<<grid, kThreads, C::SMEM, s>>>(xm, wm, args);
  return cudaGetLastError();
}

}  // namespace

cudaError_t conv3x3(const __nv_bfloat16 *x, const __nv_bfloat16 *w, int n, int h, int wd, int cin, int cout,
                    const float *bias, const __nv_bfloat16 *mask, __nv_bfloat16 *y, int mode, int *err,
                    cudaStream_t s) {
  if (n < 1 || h < 1 || wd < 1 || !x || !w || !y || !err) return cudaErrorInvalidValue;
  if ((mode == CONV_BIAS_RELU || mode == CONV_BIAS) && !bias) return cudaErrorInvalidValue;
  if (mode == CONV_MASK && !mask) return cudaErrorInvalidValue;
  if ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(w) | reinterpret_cast<uintptr_t>(y) |
       reinterpret_cast<uintptr_t>(mask)) & 15u)
    return cudaErrorMisalignedAddress;
  ConvArgs a;
  memset(&a, 0, sizeof(a));
  a.n = n;
  a.h = h;
  a.w = wd;
  a.tw = 128;
  while (a.tw > 16 && a.tw / 2 >= wd) a.tw /= 2;
  const int sub = cin == 16 ? 4 : 1;  // Cfg<cin, cout>::SUB
  a.th = sub * kTileM / a.tw;
  a.tiles_x = (wd + a.tw - 1) / a.tw;
  a.tiles_y = (h + a.th - 1) / a.th;
  long long tiles = (long long)a.tiles_x * a.tiles_y * n;
  if (tiles > (1LL << 30)) return cudaErrorInvalidValue;
  a.tiles = (int)tiles;
  a.bias = bias;
  a.mask = mask;
  a.y = y;
  a.mode = mode;
  a.err = err;
#define OPSB_CONV_CASE(CI, CO) \
  if (cin == CI && cout == CO) return launch<CI, CO>(x, w, a, s);
  OPSB_CONV_CASE(16, 16)
  OPSB_CONV_CASE(16, 32)
  OPSB_CONV_CASE(32, 16)
  OPSB_CONV_CASE(32, 32)
  OPSB_CONV_CASE(32, 64)
  OPSB_CONV_CASE(64, 32)
  OPSB_CONV_CASE(64, 64)
#undef OPSB_CONV_CASE
  return cudaErrorInvalidValue;
}

}  // namespace cnn
}  // namespace opsb
