// unet3d.cu — kernels of the learned warm start (include/unet3d.h): 3x3x3
// convolutions as implicit GEMMs on the BF16 tensor cores (mma.sync m16n8k16,
// FP32 accumulation), their data and weight gradients, 2x pooling / upsampling with
// skip concatenation, the masked MSE loss and Adam.
//
// Forward (and data-gradient) convolution: one warp computes a tile of 16
// consecutive voxels along x by all output channels.  The K loop runs over the 27
// taps and 16-channel slices of the input; A fragments are read straight from the
// channels-last activations (each thread loads the 32-bit channel pairs of two
// voxels), B fragments from the [tap][Cout][Cin] weights, both through the read-only
// cache.  Taps whose row lies outside the box are skipped warp-uniformly; voxels
// outside the row read zero.
//
// Weight gradient: dW[tap] = dY^T X_shift is a GEMM whose reduction runs over the
// voxels.  A block owns one tap, a 16-channel input slice and a chunk of voxels:
// it stages 64-voxel slabs of dY and of the shifted input in shared memory and
// feeds the MMAs with transposing ldmatrix loads; partial sums go to the FP32
// gradient with one atomic add per element and block.
#include <cuda.h>  // CUtensorMap and its enums (the encoder is fetched at run time)
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <mutex>
#include <cudaTypedefs.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/unet3d.h"

namespace {

thread_local std::string g_err;

int fail(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return 1;
}

int launched(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail("%s: %s", what, cudaGetErrorString(e));
  return 0;
}

using bf16 = __nv_bfloat16;

struct Geo {
  int n, d, h, w;
};

__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ void ldsm_x4_trans(uint32_t* r, const void* smem_row) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(smem_row);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// ---- forward convolution ------------------------------------------------------------
template <int NT>  // output channels / 8
__global__ void __launch_bounds__(128) conv_fwd_kernel(const bf16* __restrict__ in, const bf16* __restrict__ w,
                                                       const float* __restrict__ bias, bf16* __restrict__ out,
                                                       const Geo g, const int cin, const int relu,
                                                       const long long tiles) {
  const int lane = threadIdx.x & 31;
  const long long tile = (long long)blockIdx.x * 4 + (threadIdx.x >> 5);
  if (tile >= tiles) return;  // whole warp
  const int tpr = g.w / 16;
  long long row = tile / tpr;
  const int x0 = (int)(tile - row * tpr) * 16;
  const int y = (int)(row % g.h);
  row /= g.h;
  const int z = (int)(row % g.d);
  const int n = (int)(row / g.d);
  const int gid = lane >> 2, tig = lane & 3;
  constexpr int COUT = NT * 8;
  const int cw = cin / 2;  // 32-bit words per voxel
  const uint32_t* in32 = reinterpret_cast<const uint32_t*>(in);
  const uint32_t* w32 = reinterpret_cast<const uint32_t*>(w);
  float acc[NT][4];
#pragma unroll
  for (int t = 0; t < NT; t++) acc[t][0] = acc[t][1] = acc[t][2] = acc[t][3] = 0.f;
  for (int dz = -1; dz <= 1; dz++) {
    const int zz = z + dz;
    if (zz < 0 || zz >= g.d) continue;
    for (int dy = -1; dy <= 1; dy++) {
      const int yy = y + dy;
      if (yy < 0 || yy >= g.h) continue;
      const long long rbase = (((long long)n * g.d + zz) * g.h + yy) * g.w;
#pragma unroll
      for (int dx = -1; dx <= 1; dx++) {
        const int tap = ((dz + 1) * 3 + (dy + 1)) * 3 + (dx + 1);
        const int xa = x0 + gid + dx, xb = xa + 8;
        const bool va = xa >= 0 && xa < g.w, vb = xb >= 0 && xb < g.w;
        const uint32_t* pa = in32 + (rbase + (va ? xa : 0)) * cw + tig;
        const uint32_t* pb = in32 + (rbase + (vb ? xb : 0)) * cw + tig;
        const uint32_t* wt = w32 + ((long long)tap * COUT + gid) * cw + tig;
        for (int k2 = 0; k2 < cw; k2 += 8) {
          uint32_t a[4];
          a[0] = va ? __ldg(pa + k2) : 0u;
          a[1] = vb ? __ldg(pb + k2) : 0u;
          a[2] = va ? __ldg(pa + k2 + 4) : 0u;
          a[3] = vb ? __ldg(pb + k2 + 4) : 0u;
#pragma unroll
          for (int t = 0; t < NT; t++) {
            const uint32_t* wb = wt + (long long)t * 8 * cw + k2;
            const uint32_t b[2] = {__ldg(wb), __ldg(wb + 4)};
            mma_bf16(acc[t], a, b);
          }
        }
      }
    }
  }
  const long long vbase = (((long long)n * g.d + z) * g.h + y) * g.w + x0;
  uint32_t* o32 = reinterpret_cast<uint32_t*>(out);
#pragma unroll
  for (int t = 0; t < NT; t++) {
    const int co = t * 8 + 2 * tig;
    const float b0 = bias ? bias[co] : 0.f, b1 = bias ? bias[co + 1] : 0.f;
    float v0 = acc[t][0] + b0, v1 = acc[t][1] + b1, v2 = acc[t][2] + b0, v3 = acc[t][3] + b1;
    if (relu) {
      v0 = fmaxf(v0, 0.f);
      v1 = fmaxf(v1, 0.f);
      v2 = fmaxf(v2, 0.f);
      v3 = fmaxf(v3, 0.f);
    }
    o32[((vbase + gid) * COUT + co) / 2] = pack_bf16(v0, v1);
    o32[((vbase + gid + 8) * COUT + co) / 2] = pack_bf16(v2, v3);
  }
}

// ---- forward convolution on the 5th-generation tensor cores (tcgen05) ----------------
// A CTA owns 128 consecutive voxels (M = 128) and all output channels (N = Cout); the
// K loop runs over 27 taps x 16-channel slices, one tcgen05.mma (K = 16) each.  Every
// thread gathers its voxel's 16 channels of the tap's neighbour into the A tile and the
// CTA copies the tap's 16 x Cout weights into the B tile, both in the K-major
// "interleaved" core-matrix layout (8 rows x 16 bytes per core matrix); two stages, so
// the next gather overlaps the running MMA.  One thread issues the MMA and commits it
// to the stage's mbarrier; the FP32 accumulator lives in tensor memory (TMEM) and is
// read back with tcgen05.ld for the bias / ReLU / BF16 epilogue.  Every wait is
// bounded: a wait that gives up sets the error word and the CTA still frees its TMEM.
constexpr int TC_M = 128;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, K-major, no swizzle: start, leading-dimension byte
// offset (between the two 8-element K halves), stride byte offset (between 8-row
// groups), descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of kind::f16: BF16 A and B (K-major), FP32 accumulator, M x N.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void tc_mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}

// Bounded wait on an mbarrier phase: false after `polls` polls (each try_wait blocks for
// a hardware-defined interval; the default gives up after seconds).
constexpr int TC_WAIT_POLLS = 1 << 22;
__device__ __forceinline__ bool tc_mbar_wait(uint64_t* bar, uint32_t parity, int polls = TC_WAIT_POLLS) {
  const uint32_t a = smem_addr(bar);
  for (int it = 0; it < polls; it++) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// Probe of tc_mbar_wait: thread 0 initialises an mbarrier that expects one arrival, no
// MMA commits to it and nothing arrives, so the wait gives up after `polls` polls and
// the block sets the error word as a convolution CTA does.  Nothing is in flight.
__global__ void __launch_bounds__(32) tc_wait_probe_kernel(const int polls, int* err) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    tc_mbar_init(&bar);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const bool ok = tc_mbar_wait(&bar, 0u, polls);
  if (!__all_sync(0xffffffffu, ok) && threadIdx.x == 0) atomicExch(err, 1);
}

template <int COUT>
__global__ void __launch_bounds__(TC_M) conv_fwd_tc_kernel(const bf16* __restrict__ in, const bf16* __restrict__ w,
                                                           const float* __restrict__ bias, bf16* __restrict__ out,
                                                           const Geo g, const int cin, const int relu,
                                                           const long long voxels, int* err) {
  constexpr int NCOL = COUT <= 32 ? 32 : (COUT <= 64 ? 64 : 128);  // TMEM columns: a power of two >= 32
  constexpr uint32_t A_LBO = TC_M * 16, B_LBO = COUT * 16;          // bytes per K half
  __shared__ __align__(128) uint8_t sA[2][2 * A_LBO];
  __shared__ __align__(128) uint8_t sB[2][2 * B_LBO];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_base)),
                 "r"(NCOL)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    tc_mbar_init(&bar[0]);
    tc_mbar_init(&bar[1]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;

  // this thread's voxel: row `tid` of the A tile and lane `tid` of the accumulator
  const long long v = (long long)blockIdx.x * TC_M + tid;
  const bool valid = v < voxels;
  long long t = valid ? v : 0;
  const int x = (int)(t % g.w);
  t /= g.w;
  const int y = (int)(t % g.h);
  t /= g.h;
  const int z = (int)(t % g.d);
  const uint32_t a_row = (uint32_t)((tid & 7) * 16 + (tid >> 3) * 128);
  const int kcs = cin / 16, iters = 27 * kcs;
  constexpr uint32_t IDESC = umma_idesc_bf16(TC_M, COUT);
  uint32_t parity[2] = {0u, 0u};
  bool ok = true;
  int issued = 0;
  const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
  for (int it = 0; it < iters; it++) {
    const int s = it & 1;
    bool waited = true;
    if (it >= 2) {  // the MMA of iteration it-2 read this stage
      waited = tc_mbar_wait(&bar[s], parity[s]);
      parity[s] ^= 1u;
    }
    const int tap = it / kcs, kc = it - tap * kcs;
    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
    uint4 a0 = zero, a1 = zero;
    const int xx = x + dx, yy = y + dy, zz = z + dz;
    if (valid && xx >= 0 && xx < g.w && yy >= 0 && yy < g.h && zz >= 0 && zz < g.d) {
      const long long nb = v + dx + (long long)g.w * (dy + (long long)g.h * dz);
      const uint4* src = reinterpret_cast<const uint4*>(in + nb * cin + kc * 16);
      a0 = __ldg(src);
      a1 = __ldg(src + 1);
    }
    *reinterpret_cast<uint4*>(sA[s] + a_row) = a0;
    *reinterpret_cast<uint4*>(sA[s] + A_LBO + a_row) = a1;
    for (int r = tid; r < COUT * 2; r += TC_M) {
      const int co = r >> 1, kh = r & 1;
      const uint4 val = __ldg(reinterpret_cast<const uint4*>(w + ((long long)tap * COUT + co) * cin + kc * 16 + kh * 8));
      *reinterpret_cast<uint4*>(sB[s] + kh * B_LBO + (co & 7) * 16 + (co >> 3) * 128) = val;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the tensor core reads through the async proxy
    if (!__syncthreads_and(waited)) {  // a wait gave up somewhere: stop issuing (block-uniform)
      ok = false;
      break;
    }
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint64_t adesc = umma_desc(smem_addr(sA[s]), A_LBO, 128);
      const uint64_t bdesc = umma_desc(smem_addr(sB[s]), B_LBO, 128);
      const uint32_t acc = it > 0 ? 1u : 0u, mask0 = 0u;
      asm volatile(
          "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
          " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n}\n" ::"r"(tmem),
          "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(acc), "r"(mask0)
          : "memory");
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_addr(&bar[s]))
                   : "memory");
    }
    issued = it + 1;
  }
  // the last commit tracks every MMA issued before it
  bool done = true;
  if (issued > 0) done = tc_mbar_wait(&bar[(issued - 1) & 1], parity[(issued - 1) & 1]);
  ok = __syncthreads_and(ok && done) != 0;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok && valid) {
    uint32_t* o32 = reinterpret_cast<uint32_t*>(out + v * COUT);
#pragma unroll
    for (int c0 = 0; c0 < COUT; c0 += 8) {
      uint32_t r[8];
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                   : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                   : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      float f[8];
#pragma unroll
      for (int k = 0; k < 8; k++) {
        f[k] = __uint_as_float(r[k]) + (bias ? bias[c0 + k] : 0.f);
        if (relu) f[k] = fmaxf(f[k], 0.f);
      }
      const uint4 packed = make_uint4(pack_bf16(f[0], f[1]), pack_bf16(f[2], f[3]), pack_bf16(f[4], f[5]),
                                      pack_bf16(f[6], f[7]));
      *reinterpret_cast<uint4*>(o32 + c0 / 2) = packed;
    }
  } else if (ok) {
    // lanes past the last voxel still take part in the warp-wide loads
#pragma unroll
    for (int c0 = 0; c0 < COUT; c0 += 8) {
      uint32_t r[8];
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                   : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                   : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    }
  }
  if (!ok && tid == 0) atomicExch(err, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCOL) : "memory");
}

// ---- tcgen05 convolution fed by TMA --------------------------------------------------
// Same tiling as conv_fwd_tc_kernel, but the A tile of a tap is a TMA box of the
// activations: a 5-D tensor map over (C, W, H, D, N) with box {8, min(W,128),
// 128 / min(W,128), 1, 1} lands in shared memory as 128 rows of 16 bytes — exactly the
// K-major interleaved core-matrix layout (8-row groups 128 bytes apart) — and its
// out-of-range rows (the 1-voxel halo at the box faces) are filled with zeros by the
// copy engine.  Two boxes (channel halves) per tap and 16-channel slice, two more for the
// weights; one thread runs the whole pipeline (TMA issue into a ring of stages, MMA issue
// when a stage's bytes have landed, commit that frees the stage), so no CTA barrier sits
// in the K loop.  Every wait is bounded.
constexpr int TMA_STAGES = 4;

__device__ __forceinline__ void tc_mbar_expect(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
      "%6}], [%7];" ::"r"(smem_addr(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_addr(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
      : "memory");
}

template <int COUT>
__global__ void __launch_bounds__(TC_M) conv_fwd_tma_kernel(const __grid_constant__ CUtensorMap xmap,
                                                            const __grid_constant__ CUtensorMap wmap,
                                                            const float* __restrict__ bias, bf16* __restrict__ out,
                                                            const Geo g, const int cin, const int relu, int* err) {
  constexpr int NCOL = COUT <= 32 ? 32 : (COUT <= 64 ? 64 : 128);
  constexpr uint32_t A_LBO = TC_M * 16, B_LBO = COUT * 16;
  constexpr uint32_t STAGE_BYTES = 2 * A_LBO + 2 * B_LBO;
  __shared__ __align__(128) uint8_t sbuf[TMA_STAGES][STAGE_BYTES];
  __shared__ __align__(8) uint64_t full[TMA_STAGES], empty[TMA_STAGES];
  __shared__ uint32_t tmem_base;
  __shared__ int ok_s;
  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_base)),
                 "r"(NCOL)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int s = 0; s < TMA_STAGES; s++) {
      tc_mbar_init(&full[s]);
      tc_mbar_init(&empty[s]);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  // tile -> (n, z, y0, x0): 128 voxels = part of one row (W >= 128) or 128/W whole rows
  const int bw = g.w < TC_M ? g.w : TC_M, bh = TC_M / bw;
  const int tiles_x = g.w / bw, tiles_y = g.h / bh;
  long long tile = blockIdx.x;
  const int tx = (int)(tile % tiles_x);
  tile /= tiles_x;
  const int ty = (int)(tile % tiles_y);
  tile /= tiles_y;
  const int z = (int)(tile % g.d), n = (int)(tile / g.d);
  const int x0 = tx * bw, y0 = ty * bh;
  const int kcs = cin / 16, iters = 27 * kcs;
  constexpr uint32_t IDESC = umma_idesc_bf16(TC_M, COUT);
  if (tid == 0) {
    bool ok = true;
    uint32_t fpar[TMA_STAGES] = {}, epar[TMA_STAGES] = {};
    int issued_mma = 0;
    for (int it = 0; it < iters + TMA_STAGES - 1 && ok; it++) {
      if (it < iters) {  // producer: stage it % S
        const int s = it % TMA_STAGES;
        if (it >= TMA_STAGES) {  // the MMA of it - S must have released the stage
          ok = tc_mbar_wait(&empty[s], epar[s]);
          epar[s] ^= 1u;
          if (!ok) break;
        }
        const int tap = it / kcs, kc = it - tap * kcs;
        const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
        uint8_t* st = sbuf[s];
        tc_mbar_expect(&full[s], STAGE_BYTES);
        tma_load_5d(st, &xmap, kc * 16, x0 + dx, y0 + dy, z + dz, n, &full[s]);
        tma_load_5d(st + A_LBO, &xmap, kc * 16 + 8, x0 + dx, y0 + dy, z + dz, n, &full[s]);
        tma_load_3d(st + 2 * A_LBO, &wmap, kc * 16, 0, tap, &full[s]);
        tma_load_3d(st + 2 * A_LBO + B_LBO, &wmap, kc * 16 + 8, 0, tap, &full[s]);
      }
      const int j = it - (TMA_STAGES - 1);
      if (j >= 0) {  // consumer: MMA of iteration j
        const int s = j % TMA_STAGES;
        ok = tc_mbar_wait(&full[s], fpar[s]);
        fpar[s] ^= 1u;
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint64_t adesc = umma_desc(smem_addr(sbuf[s]), A_LBO, 128);
        const uint64_t bdesc = umma_desc(smem_addr(sbuf[s] + 2 * A_LBO), B_LBO, 128);
        const uint32_t acc = j > 0 ? 1u : 0u, mask0 = 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n}\n" ::"r"(tmem),
            "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(acc), "r"(mask0)
            : "memory");
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(&empty[s]))
                     : "memory");
        issued_mma = j + 1;
      }
    }
    // the last commit tracks every MMA before it; drain the ring (bounded) either way
    if (issued_mma > 0) {
      const int s = (issued_mma - 1) % TMA_STAGES;
      const bool done = tc_mbar_wait(&empty[s], epar[s]);
      ok = ok && done;
    }
    ok_s = ok && issued_mma == iters ? 1 : 0;
  }
  __syncthreads();
  const bool ok = ok_s != 0;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    const int r = tid;  // accumulator lane = tile row = voxel
    const int x = x0 + (r % bw), y = y0 + r / bw;
    const long long v = (((long long)n * g.d + z) * g.h + y) * g.w + x;
    uint32_t* o32 = reinterpret_cast<uint32_t*>(out + v * COUT);
#pragma unroll
    for (int c0 = 0; c0 < COUT; c0 += 8) {
      uint32_t q[8];
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                   : "=r"(q[0]), "=r"(q[1]), "=r"(q[2]), "=r"(q[3]), "=r"(q[4]), "=r"(q[5]), "=r"(q[6]), "=r"(q[7])
                   : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      float f[8];
#pragma unroll
      for (int k = 0; k < 8; k++) {
        f[k] = __uint_as_float(q[k]) + (bias ? bias[c0 + k] : 0.f);
        if (relu) f[k] = fmaxf(f[k], 0.f);
      }
      *reinterpret_cast<uint4*>(o32 + c0 / 2) =
          make_uint4(pack_bf16(f[0], f[1]), pack_bf16(f[2], f[3]), pack_bf16(f[4], f[5]), pack_bf16(f[6], f[7]));
    }
  } else if (tid == 0) {
    atomicExch(err, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCOL) : "memory");
}

// wt[26 - tap][ci][co] = w[tap][co][ci]
__global__ void flip_kernel(const bf16* __restrict__ w, bf16* __restrict__ wt, int cin, int cout) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int total = 27 * cin * cout;
  if (i >= total) return;
  const int ci = i % cin, co = (i / cin) % cout, tap = i / (cin * cout);
  wt[((26 - tap) * cin + ci) * cout + co] = w[i];
}

// ---- weight gradient ----------------------------------------------------------------
constexpr int BW_KV = 64;  // voxels per shared-memory slab

template <int CB>  // output channels / 16 (1, 2 or 4)
__global__ void __launch_bounds__(128) conv_bwdw_kernel(const bf16* __restrict__ in, const bf16* __restrict__ dout,
                                                        float* __restrict__ dw, const Geo g, const int cin,
                                                        const long long vox, const long long chunk) {
  constexpr int COUT = CB * 16;
  constexpr int SA = COUT + 8, SB = 16 + 8;  // padded row lengths (16-byte multiples)
  __shared__ __align__(16) bf16 sA[BW_KV * SA];
  __shared__ __align__(16) bf16 sB[BW_KV * SB];
  const int tap = blockIdx.z;
  const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
  const int ci0 = blockIdx.y * 16;
  const long long m_begin = (long long)blockIdx.x * chunk;
  const long long m_end = m_begin + chunk < vox ? m_begin + chunk : vox;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr int NWB = CB < 4 ? CB : 4;  // warps sharing the output-channel blocks
  const int cb = warp % NWB, phase = warp / NWB, nphase = 4 / NWB;
  float acc[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
  const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
  for (long long m0 = m_begin; m0 < m_end; m0 += BW_KV) {
    // dY slab: BW_KV voxels x COUT channels, 16-byte chunks
    for (int c = tid; c < BW_KV * (COUT / 8); c += 128) {
      const int i = c / (COUT / 8), part = c % (COUT / 8);
      const long long m = m0 + i;
      const uint4 v = m < m_end ? *reinterpret_cast<const uint4*>(dout + m * COUT + part * 8) : zero;
      *reinterpret_cast<uint4*>(sA + i * SA + part * 8) = v;
    }
    // shifted input slab: BW_KV voxels x 16 channels
    {
      const int i = tid >> 1, part = tid & 1;
      const long long m = m0 + i;
      uint4 v = zero;
      if (m < m_end) {
        long long t = m;
        const int x = (int)(t % g.w);
        t /= g.w;
        const int y = (int)(t % g.h);
        t /= g.h;
        const int z = (int)(t % g.d);
        const int xx = x + dx, yy = y + dy, zz = z + dz;
        if (xx >= 0 && xx < g.w && yy >= 0 && yy < g.h && zz >= 0 && zz < g.d) {
          const long long nb = m + dx + (long long)g.w * (dy + (long long)g.h * dz);
          v = *reinterpret_cast<const uint4*>(in + nb * cin + ci0 + part * 8);
        }
      }
      *reinterpret_cast<uint4*>(sB + i * SB + part * 8) = v;
    }
    __syncthreads();
    for (int k16 = phase; k16 < BW_KV / 16; k16 += nphase) {
      const int i = lane & 7, mat = lane >> 3;
      uint32_t a[4], b[4];
      ldsm_x4_trans(a, sA + (k16 * 16 + i + (mat >= 2 ? 8 : 0)) * SA + cb * 16 + ((mat & 1) ? 8 : 0));
      ldsm_x4_trans(b, sB + (k16 * 16 + i + ((mat & 1) ? 8 : 0)) * SB + (mat >> 1) * 8);
      mma_bf16(acc[0], a, b);
      mma_bf16(acc[1], a, b + 2);
    }
    __syncthreads();
  }
  const int gid = lane >> 2, tig = lane & 3;
#pragma unroll
  for (int t = 0; t < 2; t++) {
    const int co = cb * 16 + gid, ci = ci0 + t * 8 + 2 * tig;
    float* p = dw + ((long long)tap * COUT + co) * cin + ci;
    atomicAdd(p, acc[t][0]);
    atomicAdd(p + 1, acc[t][1]);
    atomicAdd(p + 8LL * cin, acc[t][2]);
    atomicAdd(p + 8LL * cin + 1, acc[t][3]);
  }
}

__global__ void bias_grad_kernel(const bf16* __restrict__ dout, float* __restrict__ db, long long voxels, int c) {
  extern __shared__ float sacc[];
  for (int k = threadIdx.x; k < c; k += blockDim.x) sacc[k] = 0.f;
  __syncthreads();
  const long long total = voxels * c;
  float s = 0.f;
  // the stride is a multiple of c, so each thread keeps one channel; threads past
  // the stride would repeat elements and stay idle
  const long long stride = (long long)gridDim.x * blockDim.x / c * c;
  const long long start = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (start < stride) {
    for (long long i = start; i < total; i += stride) s += __bfloat162float(dout[i]);
    atomicAdd(&sacc[start % c], s);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < c; k += blockDim.x) atomicAdd(db + k, sacc[k]);
}

__global__ void relu_bwd_kernel(bf16* __restrict__ dy, const bf16* __restrict__ y, long long count) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count && !(__bfloat162float(y[i]) > 0.f)) dy[i] = __float2bfloat16(0.f);
}

// ---- pooling, upsampling, concatenation ---------------------------------------------
__global__ void pool2_kernel(const bf16* __restrict__ in, bf16* __restrict__ out, Geo f, int c, long long count) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;  // count = coarse elements
  const int ch = (int)(i % c);
  long long t = i / c;
  const int W = f.w / 2, H = f.h / 2, D = f.d / 2;
  const int x = (int)(t % W);
  t /= W;
  const int y = (int)(t % H);
  t /= H;
  const int z = (int)(t % D);
  const int n = (int)(t / D);
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const long long v = (((long long)n * f.d + 2 * z + (k >> 2)) * f.h + 2 * y + ((k >> 1) & 1)) * f.w + 2 * x + (k & 1);
    s += __bfloat162float(in[v * c + ch]);
  }
  out[i] = __float2bfloat16(s * 0.125f);
}

__global__ void pool2_bwd_kernel(const bf16* __restrict__ dout, bf16* __restrict__ din, Geo f, int c, int accumulate,
                                 long long count) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;  // count = fine elements
  const int ch = (int)(i % c);
  long long t = i / c;
  const int x = (int)(t % f.w);
  t /= f.w;
  const int y = (int)(t % f.h);
  t /= f.h;
  const int z = (int)(t % f.d);
  const int n = (int)(t / f.d);
  const long long p = (((long long)n * (f.d / 2) + z / 2) * (f.h / 2) + y / 2) * (f.w / 2) + x / 2;
  float v = __bfloat162float(dout[p * c + ch]) * 0.125f;
  if (accumulate) v += __bfloat162float(din[i]);
  din[i] = __float2bfloat16(v);
}

__global__ void up2_concat_kernel(const bf16* __restrict__ low, const bf16* __restrict__ skip, bf16* __restrict__ out,
                                  Geo f, int cu, int cs, long long count) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;  // count = fine voxels * (cu + cs)
  const int ct = cu + cs;
  const int ch = (int)(i % ct);
  const long long v = i / ct;
  if (ch >= cu) {
    out[i] = skip[v * cs + (ch - cu)];
    return;
  }
  long long t = v;
  const int x = (int)(t % f.w);
  t /= f.w;
  const int y = (int)(t % f.h);
  t /= f.h;
  const int z = (int)(t % f.d);
  const int n = (int)(t / f.d);
  const long long p = (((long long)n * (f.d / 2) + z / 2) * (f.h / 2) + y / 2) * (f.w / 2) + x / 2;
  out[i] = low[p * cu + ch];
}

__global__ void up2_concat_bwd_low_kernel(const bf16* __restrict__ dcat, bf16* __restrict__ dlow, Geo f, int cu, int cs,
                                          long long count) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;  // count = coarse voxels * cu
  const int ch = (int)(i % cu);
  long long t = i / cu;
  const int W = f.w / 2, H = f.h / 2, D = f.d / 2;
  const int x = (int)(t % W);
  t /= W;
  const int y = (int)(t % H);
  t /= H;
  const int z = (int)(t % D);
  const int n = (int)(t / D);
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const long long v = (((long long)n * f.d + 2 * z + (k >> 2)) * f.h + 2 * y + ((k >> 1) & 1)) * f.w + 2 * x + (k & 1);
    s += __bfloat162float(dcat[v * (cu + cs) + ch]);
  }
  dlow[i] = __float2bfloat16(s);
}

__global__ void up2_concat_bwd_skip_kernel(const bf16* __restrict__ dcat, bf16* __restrict__ dskip, int cu, int cs,
                                           long long count) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;  // count = fine voxels * cs
  const long long v = i / cs;
  dskip[i] = dcat[v * (cu + cs) + cu + (int)(i % cs)];
}

// ---- loss and optimiser -------------------------------------------------------------
__global__ void mse_kernel(const bf16* __restrict__ out, const float* __restrict__ target,
                           const uint8_t* __restrict__ mask, const float* __restrict__ cw, bf16* __restrict__ dout,
                           double* loss, long long voxels, int cpad, int ct, double count) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double l = 0.0;
  if (v < voxels) {
    const bool on = mask[v] != 0;
    for (int c = 0; c < cpad; c++) {
      float gr = 0.f;
      if (on && c < ct) {
        const float d = __bfloat162float(out[v * cpad + c]) - target[v * ct + c];
        l += (double)cw[c] * d * d;
        gr = (float)(2.0 * cw[c] * d / count);
      }
      dout[v * cpad + c] = __float2bfloat16(gr);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0 && l != 0.0) atomicAdd(loss, l / count);
}

__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, bf16* __restrict__ wb, long long count, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (wb) wb[i] = __float2bfloat16(wi);
}

__global__ void to_bf16_kernel(const float* __restrict__ x, bf16* __restrict__ y, long long count) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) y[i] = __float2bfloat16(x[i]);
}

__global__ void from_bf16_kernel(const bf16* __restrict__ x, float* __restrict__ y, long long count) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) y[i] = __bfloat162float(x[i]);
}

// out[0] += sum (a - b)^2, out[1] += sum a^2 (FP64), for steady-state tests.
__global__ void diff_norms_kernel(const float* __restrict__ a, const float* __restrict__ b, long long count,
                                  double* out) {
  double d2 = 0.0, a2 = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (long long)gridDim.x * blockDim.x) {
    const double x = a[i], y = b[i];
    d2 += (x - y) * (x - y);
    a2 += x * x;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    d2 += __shfl_down_sync(0xffffffffu, d2, o);
    a2 += __shfl_down_sync(0xffffffffu, a2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(out, d2);
    atomicAdd(out + 1, a2);
  }
}

struct Ellipsoid {
  double center[3];
  double rot[9];  // row-major body -> world
  double semi[3];
};

// Inputs of one case: mask, approximate signed distance / 16 in [-1, 4], Re feature,
// node position; the mask uses the solver's rasteriser expression with unfused
// FP64 operations, so it matches the solver's solid flags.
__global__ void features_kernel(bf16* __restrict__ out, int nx, int ny, int nz, Ellipsoid e, float re_feature) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)nx * ny * nz;
  if (v >= n) return;
  const int x = (int)(v % nx), y = (int)((v / nx) % ny), z = (int)(v / ((long long)nx * ny));
  const double dx = __dadd_rn(x + 0.5, -e.center[0]);
  const double dy = __dadd_rn(y + 0.5, -e.center[1]);
  const double dz = __dadd_rn(z + 0.5, -e.center[2]);
  const double* r = e.rot;
  double b[3], q[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    b[k] = __dadd_rn(__dadd_rn(__dmul_rn(r[k], dx), __dmul_rn(r[3 + k], dy)), __dmul_rn(r[6 + k], dz));
    q[k] = __ddiv_rn(b[k], e.semi[k]);
  }
  const double e2 = __dadd_rn(__dadd_rn(__dmul_rn(q[0], q[0]), __dmul_rn(q[1], q[1])), __dmul_rn(q[2], q[2]));
  const double er = sqrt(e2);
  double g2 = 0.0;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const double t = b[k] / (e.semi[k] * e.semi[k]);
    g2 += t * t;
  }
  const double grad = sqrt(g2) / fmax(er, 1e-12);
  const double sdf = (er - 1.0) / fmax(grad, 1e-12);
  float f[16];
#pragma unroll
  for (int c = 0; c < 16; c++) f[c] = 0.f;
  f[0] = e2 <= 1.0 ? 1.f : 0.f;
  f[1] = fminf(fmaxf((float)(sdf / 16.0), -1.f), 4.f);
  f[2] = re_feature;
  f[3] = (float)((x + 0.5) / nx);
  f[4] = (float)((y + 0.5) / ny);
  f[5] = (float)((z + 0.5) / nz);
  uint32_t* o = reinterpret_cast<uint32_t*>(out + v * 16);
#pragma unroll
  for (int c = 0; c < 8; c++) o[c] = pack_bf16(f[2 * c], f[2 * c + 1]);
}

// out (n, 4, d, h, w) FP32 (+)= weight * the first four channels of y (n, d, h, w, 16),
// read from the mirror image in y and/or z, with the mirrored velocity components
// (channel 2 = u_y, 3 = u_z) negated: undoes a reflection of the input.
__global__ void unpack_fields_kernel(const bf16* __restrict__ y, float* __restrict__ out, Geo g, int flip_y, int flip_z,
                                     float weight, int accumulate, long long count) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;  // count = n * d * h * w
  long long t = i;
  const int x = (int)(t % g.w);
  t /= g.w;
  const int yy = (int)(t % g.h);
  t /= g.h;
  const int z = (int)(t % g.d);
  const int n = (int)(t / g.d);
  const int ys = flip_y ? g.h - 1 - yy : yy, zs = flip_z ? g.d - 1 - z : z;
  const long long src = (((long long)n * g.d + zs) * g.h + ys) * g.w + x;
  const long long plane = (long long)g.d * g.h * g.w;
  const long long v = ((long long)z * g.h + yy) * g.w + x;
#pragma unroll
  for (int c = 0; c < 4; c++) {
    float val = __bfloat162float(y[src * 16 + c]) * weight;
    if ((c == 2 && flip_y) || (c == 3 && flip_z)) val = -val;
    float* o = out + ((long long)n * 4 + c) * plane + v;
    *o = accumulate ? *o + val : val;
  }
}

// forward convolutions: 0 = mma.sync warp tiles, 1 = tcgen05 with thread-gathered tiles,
// 2 = per layer (tcgen05 when Cout >= 32: with Cout = 16 one 128-voxel gather feeds too
// small an MMA and the warp tiles are faster, measured on B200), 3 = tcgen05 with
// TMA-fed tiles where the shape allows (slower on B200 with these 16-byte-wide boxes:
// the copy engine issues one request per 16-byte row)
int g_engine = 2;

// cuTensorMapEncodeTiled from the driver (fetched once, no link against libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

// The TMA-fed kernel takes tiles of 128 voxels that are whole rows or part of one row.
bool tma_tiles_fit(int h, int w) {
  if (w >= TC_M) return w % TC_M == 0;
  return TC_M % w == 0 && h % (TC_M / w) == 0;
}
__device__ int g_tc_err;  // set by a tcgen05 kernel whose wait gave up

// Device address of g_tc_err, looked up once per device under a lock (host code cannot
// use the symbol itself as a device address).
int* tc_err_ptr() {
  static int* ptrs[64] = {nullptr};
  static std::mutex lock;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> guard(lock);
  if (!ptrs[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_tc_err) != cudaSuccess) return nullptr;
    ptrs[dev] = (int*)p;
  }
  return ptrs[dev];
}

unsigned blocks_for(long long count, int per) { return (unsigned)((count + per - 1) / per); }

bool geo_ok(int n, int d, int h, int w) { return n > 0 && d > 0 && h > 0 && w > 0; }

}  // namespace

extern "C" {

int32_t nn_abi_version(void) { return UNET3D_ABI_VERSION; }

const char* nn_last_error(void) { return g_err.c_str(); }

int32_t nn_conv3d_fwd(const void* in, const void* w, const float* bias, void* out, int32_t n, int32_t d, int32_t h,
                      int32_t wd, int32_t cin, int32_t cout, int32_t relu, void* stream) {
  if (!in || !w || !out || !geo_ok(n, d, h, wd)) return fail("nn_conv3d_fwd: null pointer or empty shape");
  if (wd % 16 || cin % 16 || cin <= 0) return fail("nn_conv3d_fwd: W (%d) and Cin (%d) must be multiples of 16", wd, cin);
  const Geo g{n, d, h, wd};
  const long long tiles = (long long)n * d * h * (wd / 16);
  const unsigned grid = blocks_for(tiles, 4);
  cudaStream_t s = (cudaStream_t)stream;
  const bf16* I = (const bf16*)in;
  const bf16* W = (const bf16*)w;
  bf16* O = (bf16*)out;
  if (g_engine == 1 || g_engine == 3 || (g_engine == 2 && cout >= 32)) {
    int* err = tc_err_ptr();
    if (!err) return fail("nn_conv3d_fwd: no device address for the error word");
    PFN_cuTensorMapEncodeTiled_v12000 enc = g_engine == 3 ? tensor_map_encoder() : nullptr;
    if (enc && tma_tiles_fit(h, wd) && cin % 16 == 0) {
      CUtensorMap xmap, wmap;
      const cuuint64_t xdim[5] = {(cuuint64_t)cin, (cuuint64_t)wd, (cuuint64_t)h, (cuuint64_t)d, (cuuint64_t)n};
      const cuuint64_t xstr[4] = {(cuuint64_t)cin * 2, (cuuint64_t)wd * cin * 2, (cuuint64_t)h * wd * cin * 2,
                                  (cuuint64_t)d * h * wd * cin * 2};
      const int bw = wd < TC_M ? wd : TC_M;
      const cuuint32_t xbox[5] = {8, (cuuint32_t)bw, (cuuint32_t)(TC_M / bw), 1, 1};
      const cuuint32_t one[5] = {1, 1, 1, 1, 1};
      const cuuint64_t wdim[3] = {(cuuint64_t)cin, (cuuint64_t)cout, 27};
      const cuuint64_t wstr[2] = {(cuuint64_t)cin * 2, (cuuint64_t)cout * cin * 2};
      const cuuint32_t wbox[3] = {8, (cuuint32_t)cout, 1};
      CUresult r1 = enc(&xmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(in), xdim, xstr, xbox, one,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      CUresult r2 = enc(&wmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(w), wdim, wstr, wbox, one,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r1 != CUDA_SUCCESS || r2 != CUDA_SUCCESS) return fail("nn_conv3d_fwd: tensor map encoding failed (%d, %d)", (int)r1, (int)r2);
      const unsigned tgrid = (unsigned)((long long)n * d * (h / (TC_M / bw)) * (wd / bw));
      switch (cout) {
        case 16: conv_fwd_tma_kernel<16><<<tgrid, TC_M, 0, s>>>(xmap, wmap, bias, O, g, cin, relu, err); break;
        case 32: conv_fwd_tma_kernel<32><<<tgrid, TC_M, 0, s>>>(xmap, wmap, bias, O, g, cin, relu, err); break;
        case 48: conv_fwd_tma_kernel<48><<<tgrid, TC_M, 0, s>>>(xmap, wmap, bias, O, g, cin, relu, err); break;
        case 64: conv_fwd_tma_kernel<64><<<tgrid, TC_M, 0, s>>>(xmap, wmap, bias, O, g, cin, relu, err); break;
        case 96: conv_fwd_tma_kernel<96><<<tgrid, TC_M, 0, s>>>(xmap, wmap, bias, O, g, cin, relu, err); break;
        default: return fail("nn_conv3d_fwd: Cout %d not in {16, 32, 48, 64, 96}", cout);
      }
      return launched("nn_conv3d_fwd (tcgen05, TMA)");
    }
    const long long vox = (long long)n * d * h * wd;
    const unsigned tgrid = blocks_for(vox, TC_M);
    switch (cout) {
      case 16: conv_fwd_tc_kernel<16><<<tgrid, TC_M, 0, s>>>(I, W, bias, O, g, cin, relu, vox, err); break;
      case 32: conv_fwd_tc_kernel<32><<<tgrid, TC_M, 0, s>>>(I, W, bias, O, g, cin, relu, vox, err); break;
      case 48: conv_fwd_tc_kernel<48><<<tgrid, TC_M, 0, s>>>(I, W, bias, O, g, cin, relu, vox, err); break;
      case 64: conv_fwd_tc_kernel<64><<<tgrid, TC_M, 0, s>>>(I, W, bias, O, g, cin, relu, vox, err); break;
      case 96: conv_fwd_tc_kernel<96><<<tgrid, TC_M, 0, s>>>(I, W, bias, O, g, cin, relu, vox, err); break;
      default: return fail("nn_conv3d_fwd: Cout %d not in {16, 32, 48, 64, 96}", cout);
    }
    return launched("nn_conv3d_fwd (tcgen05)");
  }
  switch (cout) {
    case 16: conv_fwd_kernel<2><<<grid, 128, 0, s>>>(I, W, bias, O, g, cin, relu, tiles); break;
    case 32: conv_fwd_kernel<4><<<grid, 128, 0, s>>>(I, W, bias, O, g, cin, relu, tiles); break;
    case 48: conv_fwd_kernel<6><<<grid, 128, 0, s>>>(I, W, bias, O, g, cin, relu, tiles); break;
    case 64: conv_fwd_kernel<8><<<grid, 128, 0, s>>>(I, W, bias, O, g, cin, relu, tiles); break;
    case 96: conv_fwd_kernel<12><<<grid, 128, 0, s>>>(I, W, bias, O, g, cin, relu, tiles); break;
    default: return fail("nn_conv3d_fwd: Cout %d not in {16, 32, 48, 64, 96}", cout);
  }
  return launched("nn_conv3d_fwd");
}

int32_t nn_set_conv_engine(int32_t engine) {
  if (engine < 0 || engine > 3) {
    fail("nn_set_conv_engine: engine must be 0 (mma.sync), 1 (tcgen05), 2 (per layer) or 3 (tcgen05, TMA-fed)");
    return -1;
  }
  const int prev = g_engine;
  g_engine = engine;
  g_err.clear();
  return prev;
}

int32_t nn_conv_uses_tma(int32_t h, int32_t wd, int32_t cin, int32_t cout) {
  (void)cout;
  return (g_engine == 3 && tensor_map_encoder() && tma_tiles_fit(h, wd) && cin % 16 == 0) ? 1 : 0;
}

int32_t nn_tc_status(void* stream) {
  int* err = tc_err_ptr();
  if (!err) return fail("nn_tc_status: no device address for the error word");
  int h = 0;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return launched("nn_tc_status");
  if (h) {
    cudaMemsetAsync(err, 0, sizeof(int), s);
    return fail("a tcgen05 convolution gave up waiting for its MMA (error word %d)", h);
  }
  return 0;
}

int32_t nn_wait_selftest(int32_t polls, void* stream) {
  if (polls < 1 || polls > TC_WAIT_POLLS) return fail("nn_wait_selftest: polls %d outside [1, %d]", polls, TC_WAIT_POLLS);
  int* err = tc_err_ptr();
  if (!err) return fail("nn_wait_selftest: no device address for the error word");
  tc_wait_probe_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(polls, err);
  const int rc = launched("nn_wait_selftest");
  if (rc) return rc;
  return nn_tc_status(stream);
}

int32_t nn_conv3d_flip(const void* w, void* wt, int32_t cin, int32_t cout, void* stream) {
  if (!w || !wt || cin <= 0 || cout <= 0) return fail("nn_conv3d_flip: bad arguments");
  const int total = 27 * cin * cout;
  flip_kernel<<<blocks_for(total, 256), 256, 0, (cudaStream_t)stream>>>((const bf16*)w, (bf16*)wt, cin, cout);
  return launched("nn_conv3d_flip");
}

int32_t nn_conv3d_bwd_weight(const void* in, const void* dout, float* dw, int32_t n, int32_t d, int32_t h, int32_t wd,
                             int32_t cin, int32_t cout, void* stream) {
  if (!in || !dout || !dw || !geo_ok(n, d, h, wd)) return fail("nn_conv3d_bwd_weight: null pointer or empty shape");
  if (cin % 16 || cin <= 0) return fail("nn_conv3d_bwd_weight: Cin %d must be a multiple of 16", cin);
  const long long vox = (long long)n * d * h * wd;
  const long long chunk = 4096;
  dim3 grid(blocks_for(vox, (int)chunk), (unsigned)(cin / 16), 27);
  const Geo g{n, d, h, wd};
  cudaStream_t s = (cudaStream_t)stream;
  const bf16* I = (const bf16*)in;
  const bf16* D = (const bf16*)dout;
  switch (cout) {
    case 16: conv_bwdw_kernel<1><<<grid, 128, 0, s>>>(I, D, dw, g, cin, vox, chunk); break;
    case 32: conv_bwdw_kernel<2><<<grid, 128, 0, s>>>(I, D, dw, g, cin, vox, chunk); break;
    case 64: conv_bwdw_kernel<4><<<grid, 128, 0, s>>>(I, D, dw, g, cin, vox, chunk); break;
    default: return fail("nn_conv3d_bwd_weight: Cout %d not in {16, 32, 64}", cout);
  }
  return launched("nn_conv3d_bwd_weight");
}

int32_t nn_bias_grad(const void* dout, float* db, int64_t voxels, int32_t c, void* stream) {
  if (!dout || !db || voxels <= 0 || c <= 0 || c > 256) return fail("nn_bias_grad: bad arguments");
  const long long total = voxels * c;
  unsigned grid = blocks_for(total, 256 * 16);
  if (grid > 4096) grid = 4096;
  bias_grad_kernel<<<grid, 256, c * sizeof(float), (cudaStream_t)stream>>>((const bf16*)dout, db, voxels, c);
  return launched("nn_bias_grad");
}

int32_t nn_relu_bwd(void* dy, const void* y, int64_t count, void* stream) {
  if (!dy || !y || count < 0) return fail("nn_relu_bwd: bad arguments");
  if (count == 0) return 0;
  relu_bwd_kernel<<<blocks_for(count, 256), 256, 0, (cudaStream_t)stream>>>((bf16*)dy, (const bf16*)y, count);
  return launched("nn_relu_bwd");
}

int32_t nn_pool2(const void* in, void* out, int32_t n, int32_t d, int32_t h, int32_t wd, int32_t c, void* stream) {
  if (!in || !out || !geo_ok(n, d, h, wd) || c <= 0 || d % 2 || h % 2 || wd % 2) return fail("nn_pool2: bad shape");
  const long long count = (long long)n * (d / 2) * (h / 2) * (wd / 2) * c;
  pool2_kernel<<<blocks_for(count, 256), 256, 0, (cudaStream_t)stream>>>((const bf16*)in, (bf16*)out,
                                                                          Geo{n, d, h, wd}, c, count);
  return launched("nn_pool2");
}

int32_t nn_pool2_bwd(const void* dout, void* din, int32_t n, int32_t d, int32_t h, int32_t wd, int32_t c,
                     int32_t accumulate, void* stream) {
  if (!dout || !din || !geo_ok(n, d, h, wd) || c <= 0 || d % 2 || h % 2 || wd % 2) return fail("nn_pool2_bwd: bad shape");
  const long long count = (long long)n * d * h * wd * c;
  pool2_bwd_kernel<<<blocks_for(count, 256), 256, 0, (cudaStream_t)stream>>>((const bf16*)dout, (bf16*)din,
                                                                              Geo{n, d, h, wd}, c, accumulate, count);
  return launched("nn_pool2_bwd");
}

int32_t nn_up2_concat(const void* low, const void* skip, void* out, int32_t n, int32_t d, int32_t h, int32_t wd,
                      int32_t cu, int32_t cs, void* stream) {
  if (!low || !skip || !out || !geo_ok(n, d, h, wd) || cu <= 0 || cs <= 0 || d % 2 || h % 2 || wd % 2)
    return fail("nn_up2_concat: bad shape");
  const long long count = (long long)n * d * h * wd * (cu + cs);
  up2_concat_kernel<<<blocks_for(count, 256), 256, 0, (cudaStream_t)stream>>>(
      (const bf16*)low, (const bf16*)skip, (bf16*)out, Geo{n, d, h, wd}, cu, cs, count);
  return launched("nn_up2_concat");
}

int32_t nn_up2_concat_bwd(const void* dcat, void* dlow, void* dskip, int32_t n, int32_t d, int32_t h, int32_t wd,
                          int32_t cu, int32_t cs, void* stream) {
  if (!dcat || !dlow || !dskip || !geo_ok(n, d, h, wd) || cu <= 0 || cs <= 0 || d % 2 || h % 2 || wd % 2)
    return fail("nn_up2_concat_bwd: bad shape");
  cudaStream_t s = (cudaStream_t)stream;
  const long long cl = (long long)n * (d / 2) * (h / 2) * (wd / 2) * cu;
  up2_concat_bwd_low_kernel<<<blocks_for(cl, 256), 256, 0, s>>>((const bf16*)dcat, (bf16*)dlow, Geo{n, d, h, wd}, cu,
                                                                 cs, cl);
  const long long cf = (long long)n * d * h * wd * cs;
  up2_concat_bwd_skip_kernel<<<blocks_for(cf, 256), 256, 0, s>>>((const bf16*)dcat, (bf16*)dskip, cu, cs, cf);
  return launched("nn_up2_concat_bwd");
}

int32_t nn_mse(const void* out, const float* target, const uint8_t* mask, const float* cw, void* dout, double* loss,
               int64_t voxels, int32_t cpad, int32_t ct, double count, void* stream) {
  if (!out || !target || !mask || !cw || !dout || !loss || voxels <= 0 || ct <= 0 || ct > cpad || !(count > 0))
    return fail("nn_mse: bad arguments");
  mse_kernel<<<blocks_for(voxels, 256), 256, 0, (cudaStream_t)stream>>>((const bf16*)out, target, mask, cw,
                                                                         (bf16*)dout, loss, voxels, cpad, ct, count);
  return launched("nn_mse");
}

int32_t nn_adam(float* w, const float* g, float* m, float* v, void* wb, int64_t count, float lr, float beta1,
                float beta2, float eps, int32_t t, void* stream) {
  if (!w || !g || !m || !v || count < 0 || t < 1) return fail("nn_adam: bad arguments");
  if (count == 0) return 0;
  const float c1 = 1.f - powf(beta1, (float)t), c2 = 1.f - powf(beta2, (float)t);
  adam_kernel<<<blocks_for(count, 256), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, (bf16*)wb, count, lr, beta1, beta2,
                                                                         eps, c1, c2);
  return launched("nn_adam");
}

int32_t nn_diff_norms(const float* a, const float* b, int64_t count, double* out, void* stream) {
  if (!a || !b || !out || count < 0) return fail("nn_diff_norms: bad arguments");
  if (count == 0) return 0;
  unsigned grid = blocks_for(count, 256 * 8);
  if (grid > 2048) grid = 2048;
  diff_norms_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(a, b, count, out);
  return launched("nn_diff_norms");
}

int32_t nn_features_ellipsoid(void* out, int32_t nx, int32_t ny, int32_t nz, const double* center,
                              const double* rot, const double* semi, float re_feature, void* stream) {
  if (!out || !center || !rot || !semi || nx <= 0 || ny <= 0 || nz <= 0) return fail("nn_features_ellipsoid: bad arguments");
  Ellipsoid e{};
  for (int k = 0; k < 3; k++) {
    e.center[k] = center[k];
    e.semi[k] = semi[k];
  }
  for (int k = 0; k < 9; k++) e.rot[k] = rot[k];
  const long long n = (long long)nx * ny * nz;
  features_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>((bf16*)out, nx, ny, nz, e, re_feature);
  return launched("nn_features_ellipsoid");
}

int32_t nn_unpack_fields(const void* y, float* out, int32_t n, int32_t d, int32_t h, int32_t wd, int32_t flip_y,
                         int32_t flip_z, float weight, int32_t accumulate, void* stream) {
  if (!y || !out || !geo_ok(n, d, h, wd)) return fail("nn_unpack_fields: bad arguments");
  const long long count = (long long)n * d * h * wd;
  unpack_fields_kernel<<<blocks_for(count, 256), 256, 0, (cudaStream_t)stream>>>(
      (const bf16*)y, out, Geo{n, d, h, wd}, flip_y, flip_z, weight, accumulate, count);
  return launched("nn_unpack_fields");
}

int32_t nn_to_bf16(const float* x, void* y, int64_t count, void* stream) {
  if (!x || !y || count < 0) return fail("nn_to_bf16: bad arguments");
  if (count == 0) return 0;
  to_bf16_kernel<<<blocks_for(count, 256), 256, 0, (cudaStream_t)stream>>>(x, (bf16*)y, count);
  return launched("nn_to_bf16");
}

int32_t nn_from_bf16(const void* x, float* y, int64_t count, void* stream) {
  if (!x || !y || count < 0) return fail("nn_from_bf16: bad arguments");
  if (count == 0) return 0;
  from_bf16_kernel<<<blocks_for(count, 256), 256, 0, (cudaStream_t)stream>>>((const bf16*)x, y, count);
  return launched("nn_from_bf16");
}

}  // extern "C"
