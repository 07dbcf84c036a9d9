// 3x3x3 convolution forward on the 5th-generation tensor cores (tcgen05.mma, BF16 operands,
// FP32 accumulators in tensor memory): the learned smoother's layers, a K = 27 Ci contraction
// per output voxel.
//
// Activations are channels-last BF16, [B][Z][Y][X][Ci], so that the 8 channels of one voxel are
// one 16-byte row of a UMMA core matrix and the input moves with plain 16-byte cp.async copies.
//
// Implicit GEMM without an im2col copy.  A tile is M = 128 output voxels (one z-plane, 16 y-rows
// of 8 x-points) for all N = Co output channels (padded to a multiple of 32).  A CTA owns a
// column of tiles (b, y block, x block, a z segment) and walks it in z.  Its input halo planes
// (18 y-rows x 10 x-points x Ci) sit in shared memory as [y][channel chunk of 8][x][8 channels]
// in a ring of four: the MMAs of tile z read planes z - 1, z, z + 1 while the fourth slot takes
// plane z + 2.  In that layout the A operand of every tap (dz, dy, dx) and pair of channel
// chunks is a strided view of a plane with the canonical K-major, non-swizzled UMMA form: the 8
// rows of a core matrix are 8 consecutive x (16 bytes apart), the next 8 rows are the next
// y-row (stride byte offset = one plane row), the next 8 channels are the next chunk (leading
// byte offset = one chunk of 10 x-points).  So the 27 Ci / 16 K-steps of a tile are that many
// tcgen05.mma instructions with shifted start addresses.  The B operand (weights, packed once
// as [tap * Ci/8 + ci/8][co][8] BF16) stays in shared memory for the whole persistent CTA.
//
// Pipeline per z step, two TMEM accumulators: thread 0 issues the MMAs of tile z into
// accumulator z % 2 and commits them to mbarrier z % 2; all threads wait (bounded) for tile
// z - 1, start the cp.async copies of plane z + 2 into the slot tile z - 1 has released, read
// tile z - 1 out of TMEM (tcgen05.ld 32x32b; warps w and w + 4 share lanes 32 (w % 4)..+31 and
// split the columns), add the bias, apply ReLU and store; then wait for the copies and meet at
// one barrier.  The MMAs of tile z run under the copies and the epilogue.
//
// Descriptor encodings (shared-memory matrix descriptor and instruction descriptor of
// tcgen05.mma kind::f16) follow the PTX ISA for sm_100a.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "tcgen05_ops.cuh"

namespace grico {
namespace tc {

constexpr int kTY = 16, kTX = 8;              // output tile: 1 z-plane x 16 y x 8 x = M 128
constexpr int kHY = kTY + 2, kHX = kTX + 2;   // halo rows and points per row
constexpr int kM = kTY * kTX;                 // 128
constexpr int kWorkers = 256;                 // eight warps: halo copies and the epilogue
constexpr int kThreads = kWorkers + 32;       // and one warp that issues the MMAs
constexpr int kRing = 5;                      // halo planes: three under the MMAs, one loading, one draining

// N of the MMA: Co rounded up to a multiple of 32 (the padded columns carry zero weights)
__host__ __device__ inline int conv_tc_npad(int Co) { return (Co + 31) / 32 * 32; }
// TMEM columns of the two accumulators (a power of two, at least 32)
__host__ __device__ inline uint32_t conv_tc_tmem_cols(int Co) {
  const int n = 2 * conv_tc_npad(Co);
  return n <= 64 ? 64u : (n <= 128 ? 128u : 256u);
}
inline size_t conv_tc_plane_bytes(int Ci) { return size_t(kHY) * (Ci / 8) * kHX * 16; }
// packed weights, BF16 [27 Ci/8][Npad][8]
inline size_t conv_tc_weight_bytes(int Ci, int Co) { return size_t(27) * (Ci / 8) * conv_tc_npad(Co) * 16; }
// dynamic shared memory: 128 bytes for the mbarriers and the TMEM address, 512 for the bias,
// the halo ring, the weights
inline size_t conv_tc_smem_bytes(int Ci, int Co) {
  return 640 + kRing * conv_tc_plane_bytes(Ci) + conv_tc_weight_bytes(Ci, Co);
}
// shapes the kernel serves: Ci = 16, 32, 48 or 64 (K = 16 per MMA; the kernel is compiled per
// Ci), Co up to 128, the shared memory within the 227 KB of one CTA
inline bool conv_tc_supported(int Ci, int Co) {
  return Ci >= 16 && Ci <= 64 && Ci % 16 == 0 && Co >= 1 && Co <= 128 &&
         conv_tc_smem_bytes(Ci, Co) <= size_t(227) * 1024;
}

// wp[((tap * Ci/8 + ci/8) * Npad + co) * 8 + ci % 8] = bf16(w[co][ci][tap]), zero for co >= Co
__global__ void conv_tc_pack_weights(const float* __restrict__ w, __nv_bfloat16* __restrict__ wp, int Ci, int Co,
                                     int Npad) {
  const int n = 27 * Ci * Npad;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int e = i % 8;
    int r = i / 8;
    const int co = r % Npad;
    r /= Npad;
    const int ci = (r % (Ci / 8)) * 8 + e, tap = r / (Ci / 8);
    wp[i] = __float2bfloat16(co < Co ? w[(size_t(co) * Ci + ci) * 27 + tap] : 0.0f);
  }
}

// y[b, v, co] = act(bias[co] + sum_{ci, k} w[co, ci, k] x[b, v + off(k), ci]), k = 9 kz + 3 ky + kx,
// off(k) = (kz - 1, ky - 1, kx - 1), zero padding.  x: BF16 [B][Z][Y][X][8 CC] (16-byte aligned);
// wp: packed weights (conv_tc_pack_weights); y: BF16 [B][Z][Y][X][Co] (out_cf = 0, Co a
// multiple of 8) or FP32 [B][Co][Z][Y][X] (out_cf = 1).  Work items are (b, y block, x block,
// z segment of seglen planes), x block fastest; persistent CTAs take items blockIdx.x,
// blockIdx.x + gridDim.x, ...  Warps 0..7 copy the halo and run the epilogue, warp 8 issues the
// MMAs; one barrier per z step.  err[0] is set when an mbarrier wait gives up.
template <int CC>
__global__ void __launch_bounds__(kThreads) conv3d_cl_tc(const __nv_bfloat16* __restrict__ x,
                                                        const __nv_bfloat16* __restrict__ wp,
                                                        const float* __restrict__ bias, void* __restrict__ y,
                                                        int out_cf, int B, int Co, int Z, int Y, int X, int seglen,
                                                        int relu, int* __restrict__ err) {
  constexpr int Ci = 8 * CC;
  constexpr uint32_t kPlane = uint32_t(kHY * CC * kHX * 16);
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);  // bar[0], bar[1]: MMAs of even / odd tiles done
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + 16);
  float* bias_s = reinterpret_cast<float*>(smem + 128);
  unsigned char* ring = smem + 640;
  const int Npad = conv_tc_npad(Co);
  unsigned char* wsm = ring + kRing * kPlane;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const uint32_t ncols = conv_tc_tmem_cols(Co);

  {
    const uint4* src = reinterpret_cast<const uint4*>(wp);
    uint4* dst = reinterpret_cast<uint4*>(wsm);
    for (int i = tid; i < 27 * CC * Npad; i += kThreads) dst[i] = src[i];
    for (int c = tid; c < Npad; c += kThreads) bias_s[c] = (bias && c < Co) ? bias[c] : 0.0f;
  }
  if (warp == 0) tmem_alloc(tslot, ncols);
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
  }
  fence_async_smem();  // the weights are read by the tensor cores (async proxy)
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tslot;
  const uint32_t ring_s = smem_u32(ring);
  const uint32_t idesc = idesc_bf16(kM, Npad);
  // descriptors of the first A view (ring slot 0, tap 0, chunk 0) and the first B chunk; every
  // other view adds its offset / 16 to the start-address field (addresses stay below 2^18)
  const uint64_t adesc0 = smem_desc(ring_s, kHX * 16, CC * kHX * 16);
  const uint64_t bdesc0 = smem_desc(smem_u32(wsm), Npad * 16, 128);

  const int nty = (Y + kTY - 1) / kTY, ntx = (X + kTX - 1) / kTX, nseg = (Z + seglen - 1) / seglen;
  const int64_t items = int64_t(B) * nty * ntx * nseg;
  const int64_t vol = int64_t(Z) * Y * X;
  uint32_t ph0 = 0, ph1 = 0;  // parity of the next completion of bar[0], bar[1] (workers)
  int pending = 0;            // bit k: a commit to bar[k] not yet waited for
  int fail = 0;

  for (int64_t it = blockIdx.x; it < items && !fail; it += gridDim.x) {
    const int tx = int(it % ntx), ty = int((it / ntx) % nty);
    const int seg = int((it / (int64_t(ntx) * nty)) % nseg);
    const int b = int(it / (int64_t(ntx) * nty * nseg));
    const int x0 = tx * kTX, y0 = ty * kTY;
    const int z0 = seg * seglen, z1 = min(Z, z0 + seglen);
    const __nv_bfloat16* xb = x + int64_t(b) * vol * Ci;
    // cp.async of halo plane p (zeros outside the grid) into ring slot (p + kRing) % kRing, by
    // the worker warps; consecutive threads copy consecutive 16-byte chunks of a row of voxels
    auto load_plane = [&](int p) {
      const uint32_t dst0 = ring_s + uint32_t((p + kRing) % kRing) * kPlane;
      const bool zin = p >= 0 && p < Z;
#pragma unroll 1
      for (int e = tid; e < kHY * kHX * CC; e += kWorkers) {
        const int j = e % CC, r = e / CC;
        const int xx = r % kHX, yy = r / kHX;
        const int gy = y0 + yy - 1, gx = x0 + xx - 1;
        const bool in = zin && gy >= 0 && gy < Y && gx >= 0 && gx < X;
        const __nv_bfloat16* src = in ? xb + ((int64_t(p) * Y + gy) * X + gx) * Ci + j * 8 : x;
        cp_async16(dst0 + uint32_t(((yy * CC + j) * kHX + xx) * 16), src, in ? 16u : 0u);
      }
    };
    if (warp < 8) {
      load_plane(z0 - 1);
      load_plane(z0);
      load_plane(z0 + 1);
      cp_async_wait_all();
      fence_async_smem();
    }
    __syncthreads();
    // step z: warp 8 issues tile z (planes z - 1 .. z + 1, accumulator z % 2) while the workers
    // copy plane z + 2 (into the slot of plane z - 3, whose last reader, tile z - 2, is done) and
    // drain tile z - 1
    for (int z = z0; z <= z1; ++z) {
      const int i = z - z0;
      if (warp == 8) {
        if (z < z1 && lane == 0) {
          fence_after_sync();
          const uint32_t acc = tmem + uint32_t((i & 1) * Npad);
          uint32_t sl[3];
#pragma unroll
          for (int dz = 0; dz < 3; ++dz) sl[dz] = uint32_t((z - 1 + dz + kRing) % kRing) * (kPlane >> 4);
#pragma unroll
          for (int tap = 0; tap < 27; ++tap) {
            const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
#pragma unroll
            for (int k = 0; k < CC / 2; ++k) {
              const uint64_t ad = adesc0 + uint64_t(sl[dz] + uint32_t((dy * CC + 2 * k) * kHX + dx));
              const uint64_t bd = bdesc0 + uint64_t(uint32_t((tap * CC + 2 * k) * Npad));
              mma_bf16(acc, ad, bd, idesc, (tap | k) ? 1u : 0u);
            }
          }
          mma_commit(&bar[i & 1]);
        }
      } else {
        if (z + 1 < z1) load_plane(z + 2);
        if (z > z0) {
          // tile z - 1: bounded wait, then TMEM lanes (tile rows) 32 (w % 4) .. + 31, columns
          // 16 (w / 4) + 32 c
          const int pb = (i - 1) & 1;
          const bool done = mbar_wait(&bar[pb], pb ? ph1 : ph0);
          fail |= done ? 0 : 1;
          fence_after_sync();
          const int zo = z - 1, q = warp & 3;
          const int m = 32 * q + lane;
          const int gy = y0 + m / kTX, gx = x0 + m % kTX;
          const bool store = done && gy < Y && gx < X;
          const int64_t v = (int64_t(zo) * Y + gy) * X + gx;
          for (int c0 = (warp >> 2) * 16; c0 < Npad; c0 += 32) {
            uint32_t r[16];
            __syncwarp();
            tmem_ld16(tmem + (uint32_t(32 * q) << 16) + uint32_t(pb * Npad + c0), r);
            if (store && c0 < Co) {
              float f[16];
#pragma unroll
              for (int c = 0; c < 16; ++c) {
                const float val = __uint_as_float(r[c]) + bias_s[c0 + c];
                f[c] = relu ? fmaxf(val, 0.0f) : val;
              }
              if (out_cf) {
                float* yo = static_cast<float*>(y) + (int64_t(b) * Co + c0) * vol + v;
#pragma unroll
                for (int c = 0; c < 16; ++c)
                  if (c0 + c < Co) yo[c * vol] = f[c];
              } else {
                __nv_bfloat16* yo = static_cast<__nv_bfloat16*>(y) + (int64_t(b) * vol + v) * Co + c0;
                if (c0 + 16 <= Co) {
                  uint32_t pw[8];
#pragma unroll
                  for (int c = 0; c < 8; ++c) {
                    const __nv_bfloat162 h2 = __floats2bfloat162_rn(f[2 * c], f[2 * c + 1]);
                    pw[c] = *reinterpret_cast<const uint32_t*>(&h2);
                  }
                  reinterpret_cast<uint4*>(yo)[0] = make_uint4(pw[0], pw[1], pw[2], pw[3]);
                  reinterpret_cast<uint4*>(yo)[1] = make_uint4(pw[4], pw[5], pw[6], pw[7]);
                } else {
#pragma unroll
                  for (int c = 0; c < 16; ++c)
                    if (c0 + c < Co) yo[c] = __float2bfloat16(f[c]);
                }
              }
            }
          }
        }
        cp_async_wait_all();
        fence_async_smem();  // plane z + 2 is read by the tensor cores from step z + 1 on
      }
      fence_before_sync();
      fail = __syncthreads_or(fail);  // one decision for the whole CTA
      if (z < z1) pending |= 1 << (i & 1);
      if (fail) break;
      if (z > z0) {
        const int pb = (i - 1) & 1;
        if (pb) ph1 ^= 1u;
        else ph0 ^= 1u;
        pending &= ~(1 << pb);
      }
    }
  }
  if (fail) {
    if (tid == 0) atomicExch(err, 1);
    // let MMAs still in flight finish (bounded) before the accumulators are freed
    if (pending & 1) mbar_wait(&bar[0], ph0);
    if (pending & 2) mbar_wait(&bar[1], ph1);
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (warp == 0) tmem_dealloc(tmem, ncols);
}

// z planes per work item: the segment length that minimises (waves of items) x (planes + 2),
// the 2 standing for the three planes a segment loads before its first MMA
inline int conv_tc_seglen(int B, int Z, int Y, int X, int ctas) {
  const int64_t columns = int64_t(B) * ((Y + kTY - 1) / kTY) * ((X + kTX - 1) / kTX);
  int best = Z;
  int64_t best_cost = -1;
  for (int nseg = 1; nseg <= Z; ++nseg) {
    const int len = (Z + nseg - 1) / nseg;
    const int64_t items = columns * ((Z + len - 1) / len);
    const int64_t cost = ((items + ctas - 1) / ctas) * (len + 2);
    if (best_cost < 0 || cost < best_cost) {
      best_cost = cost;
      best = len;
    }
  }
  return best;
}

}  // namespace tc
}  // namespace grico
