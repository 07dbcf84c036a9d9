// 3x3x3 convolution forward on the 5th-generation tensor cores (tcgen05.mma, BF16 operands,
// FP32 accumulators in tensor memory): the learned smoother's 32-channel layers, a K = 27 Ci
// contraction per output voxel.
//
// Implicit GEMM without an im2col copy.  A CTA computes an M = 128 tile of output voxels (one
// z-plane, 16 y-rows of 8 x-points) for all N = Co output channels.  The input halo of the tile
// (3 z-planes x 18 y-rows x 10 x-points x Ci channels) sits in shared memory in BF16 as
// [z][y][channel chunk of 8][x][8 channels].  In that layout the A operand of every tap
// (dz, dy, dx) and pair of channel chunks is a strided view of the halo that already has the
// canonical K-major, non-swizzled UMMA form: the 8 rows of a core matrix are 8 consecutive x
// (16 bytes apart), the next 8 rows are the next y-row (stride byte offset = one halo row), the
// next 8 channels are the next chunk (leading byte offset = one chunk of 10 x-points).  So the
// 27 Ci / 16 K-steps are that many tcgen05.mma instructions with shifted start addresses.  The
// B operand (weights, K-major: [tap * Ci/8 + ci/8][co][8]) is converted to BF16 once per
// persistent CTA.  One thread issues the MMAs and commits them to an mbarrier; after a bounded
// wait the four warps read their 32 TMEM lanes (tcgen05.ld 32x32b), add the bias, apply ReLU
// and store.
//
// Descriptor encodings (shared-memory matrix descriptor and instruction descriptor of
// tcgen05.mma kind::f16) follow the PTX ISA for sm_100a.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "cnn_kernels.cuh"

namespace grico {
namespace tc {

constexpr int kTY = 16, kTX = 8;              // output tile: 1 z-plane x 16 y x 8 x = M 128
constexpr int kHY = kTY + 2, kHX = kTX + 2;   // halo rows and points per row
constexpr int kM = kTY * kTX;                 // 128
constexpr int kThreads = 128;                 // four warps: one quarter of the TMEM lanes each
constexpr uint32_t kSpinLimit = 1u << 22;     // bounded mbarrier wait (try_wait iterations)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// tcgen05 shared-memory matrix descriptor: start address, leading and stride byte offsets (all
// >> 4), version 1 (sm_100), no swizzle, base offset 0
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
         (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}

// instruction descriptor of tcgen05.mma kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// true once the phase with parity `phase` has completed; false after kSpinLimit tries
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase) {
  const uint32_t addr = smem_u32(bar);
  for (uint32_t i = 0; i < kSpinLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(addr), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 consecutive FP32 columns of this warp's 32 TMEM lanes (lane = row of the tile)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
        "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// dynamic shared memory of conv3d_fwd_tc: 128 bytes for the mbarrier and the TMEM address, the
// halo [3][kHY][Ci/8][kHX][8] and the weights [27 Ci/8][Co][8], both BF16
inline size_t conv_tc_smem_bytes(int Ci, int Co) {
  return 128 + size_t(3) * kHY * (Ci / 8) * kHX * 16 + size_t(27) * (Ci / 8) * Co * 16;
}

// shapes the kernel serves: Ci a multiple of 16, Co a multiple of 32 up to 128 (TMEM columns),
// the shared memory within the 227 KB of one CTA
inline bool conv_tc_supported(int Ci, int Co) {
  return Ci >= 16 && Ci % 16 == 0 && Co >= 32 && Co <= 128 && Co % 32 == 0 &&
         conv_tc_smem_bytes(Ci, Co) <= size_t(227) * 1024;
}

// y[b, co, v] = act(bias[co] + sum_{ci, k} w[co, ci, k] x[b, ci, v + off(k)]), k = 9 kz + 3 ky + kx,
// off(k) = (kz - 1, ky - 1, kx - 1); persistent CTAs of kThreads threads walk the tiles
// (b, z, 16-row y block, 8-point x block).  err[0] is set when an mbarrier wait gives up.
template <typename TIn, typename TOut>
__global__ void __launch_bounds__(kThreads) conv3d_fwd_tc(const TIn* __restrict__ x, const float* __restrict__ w,
                                                         const float* __restrict__ bias, TOut* __restrict__ y,
                                                         int B, int Ci, int Co, int Z, int Y, int X, int relu,
                                                         int* __restrict__ err) {
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + 8);
  __nv_bfloat16* halo = reinterpret_cast<__nv_bfloat16*>(smem + 128);
  const int CC = Ci / 8;                                  // channel chunks of 8
  __nv_bfloat16* wt = halo + size_t(3) * kHY * CC * kHX * 8;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const uint32_t ncols = Co <= 32 ? 32u : (Co <= 64 ? 64u : 128u);

  // B operand: weight (co, ci, tap) -> K-chunk tap * CC + ci / 8, row co, element ci % 8
  for (int i = tid; i < Co * Ci * 27; i += kThreads) {
    const int co = i / (Ci * 27), ci = (i / 27) % Ci, tap = i % 27;
    wt[(size_t(tap * CC + ci / 8) * Co + co) * 8 + (ci % 8)] = __float2bfloat16(w[i]);
  }
  if (warp == 0) tmem_alloc(tslot, ncols);
  if (tid == 0) mbar_init(bar, 1);
  fence_async_smem();  // the weights are read by the tensor cores (async proxy)
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tslot;
  const uint32_t halo_s = smem_u32(halo), wt_s = smem_u32(wt);
  const uint32_t idesc = idesc_bf16(kM, Co);
  const int ksteps = 27 * Ci / 16;

  const int nty = (Y + kTY - 1) / kTY, ntx = (X + kTX - 1) / kTX;
  const int64_t tiles = int64_t(B) * Z * nty * ntx;
  const int64_t vol = int64_t(Z) * Y * X;
  uint32_t phase = 0;
  bool ok = true;
  for (int64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
    const int x0 = int(t % ntx) * kTX;
    const int y0 = int((t / ntx) % nty) * kTY;
    const int z = int((t / (int64_t(ntx) * nty)) % Z);
    const int b = int(t / (int64_t(ntx) * nty * Z));
    // halo of the tile, zero outside the grid: [dz][yy][ci / 8][xx][ci % 8]
    for (int i = tid; i < 3 * kHY * Ci * kHX; i += kThreads) {
      const int xx = i % kHX;
      int r = i / kHX;
      const int ci = r % Ci;
      r /= Ci;
      const int yy = r % kHY, dz = r / kHY;
      const int gz = z + dz - 1, gy = y0 + yy - 1, gx = x0 + xx - 1;
      float v = 0.0f;
      if (gz >= 0 && gz < Z && gy >= 0 && gy < Y && gx >= 0 && gx < X)
        v = to_f(x[(int64_t(b) * Ci + ci) * vol + (int64_t(gz) * Y + gy) * X + gx]);
      halo[(size_t((dz * kHY + yy) * CC + ci / 8) * kHX + xx) * 8 + (ci % 8)] = __float2bfloat16(v);
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      fence_after_sync();
      for (int s = 0; s < ksteps; ++s) {
        const int tap = s / (Ci / 16), j = (s % (Ci / 16)) * 2;
        const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
        const uint32_t a = halo_s + uint32_t((((dz * kHY + dy) * CC + j) * kHX + dx) * 16);
        const uint32_t bb = wt_s + uint32_t(2 * s * Co * 16);
        mma_bf16(tmem, smem_desc(a, kHX * 16, CC * kHX * 16), smem_desc(bb, Co * 16, 128), idesc, s > 0 ? 1u : 0u);
      }
      mma_commit(bar);
    }
    // one decision for the whole CTA, so that no thread leaves while others reach a barrier
    ok = __syncthreads_and(mbar_wait(bar, phase) ? 1 : 0) != 0;
    phase ^= 1u;
    if (!ok) {
      if (tid == 0) atomicExch(err, 1);
      break;
    }
    fence_after_sync();
    // epilogue: warp w owns tile rows (TMEM lanes) 32 w .. 32 w + 31
    const int m = 32 * warp + lane;
    const int gy = y0 + m / kTX, gx = x0 + m % kTX;
    const bool store = gy < Y && gx < X;
    for (int c0 = 0; c0 < Co; c0 += 32) {
      uint32_t v[32];
      tmem_ld32(tmem + (uint32_t(32 * warp) << 16) + uint32_t(c0), v);
      if (store) {
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          float val = __uint_as_float(v[c]) + (bias ? bias[c0 + c] : 0.0f);
          if (relu) val = val > 0.0f ? val : 0.0f;
          y[(int64_t(b) * Co + c0 + c) * vol + (int64_t(z) * Y + gy) * X + gx] = from_f<TOut>(val);
        }
      }
    }
    fence_before_sync();
    __syncthreads();  // the TMEM accumulator and the halo are free for the next tile
  }
  if (!ok) mbar_wait(bar, phase ^ 1u);  // let MMAs still in flight finish (bounded) before freeing TMEM
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (warp == 0) tmem_dealloc(tmem, ncols);
}

}  // namespace tc
}  // namespace grico
