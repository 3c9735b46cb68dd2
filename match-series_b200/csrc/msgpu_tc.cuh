// msgpu_tc.cuh -- the warm start's forward 3x3 convolutions on the
// fifth-generation tensor cores (tcgen05, sm_100a).
//
// k_conv_tc computes the same implicit GEMM as k_conv (msgpu_unet.cuh):
// out[node][co] = sum over (tap, ci) of in[src(node, tap)][ci] * w[co][(tap, ci)],
// for a tile of 128 output nodes x BN output channels.  The operands are
// staged in shared memory in the tensor core's canonical K-major layout
// without swizzle: the 16-byte unit (row r, K chunk c of 8 elements) at
// (c * rows + r) * 16 bytes, so one unit is 8 channels of one node (NHWC) and
// is gathered by one 16-byte cp.async; a stage holds 64 K elements (8 chunks)
// of A (128 rows) and of B (BN rows), four stages in flight.  One thread
// issues tcgen05.mma (kind::f16, bf16 operands, fp32 accumulation, M = 128,
// N = BN, K = 16 per instruction) into a TMEM accumulator of BN columns;
// tcgen05.commit signals a stage's mbarrier when the MMAs reading it are
// done, which frees it for the next gather.  The epilogue reads each warp's
// 32 TMEM lanes (rows) with tcgen05.ld and applies bias, accumulation, ReLU
// and mask as k_conv does.
//
// Every mbarrier wait is bounded (kTcWaitNs of the global timer); a wait that
// runs out sets the error word, the block drains its copies, frees its TMEM
// and returns.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "msgpu_unet.cuh"

namespace msg {
namespace unet {

constexpr int kTcBM = 128;      // output nodes per tile (TMEM lanes)
constexpr int kTcBK = 64;       // K elements per stage (four MMAs)
constexpr int kTcStages = 4;
constexpr unsigned long long kTcWaitNs = 1000000000ull;   // 1 s

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long tc_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Waits for the completion of the phase with the given parity, at most
// kTcWaitNs; false when the wait ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = tc_now();
  for (;;) {
    if (mbar_try_wait(bar, parity)) return true;
    if (tc_now() - t0 > kTcWaitNs) return false;
  }
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Shared-memory matrix descriptor: K-major, no swizzle; lbo = bytes between
// the two 8-element K chunks of an MMA, sbo = bytes between 8-row groups.
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: bf16 x bf16 -> fp32, both K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t tc_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTcBM >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// 16 consecutive fp32 columns of this thread's TMEM lane
__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

template <int BN>
__host__ __device__ constexpr int tc_cols() { return BN < 32 ? 32 : BN; }
template <int BN>
__host__ __device__ constexpr size_t tc_stage_bytes() { return (size_t)16 * 8 * (kTcBM + BN); }
template <int BN>
constexpr size_t conv_tc_smem_bytes() {
  return kTcStages * tc_stage_bytes<BN>() + 128;   // + mbarriers and the TMEM address
}

// Forward convolution (mode 0; stride 1 or 2) on the tensor cores; grid
// (ceil(total / 128), rows / BN), 128 threads.  err: set to 1 when a wait
// runs out.
template <int BN>
__global__ void __launch_bounds__(128) k_conv_tc(ConvArgs a, int* err) {
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  const int tid = threadIdx.x, warp = tid >> 5;
  constexpr uint32_t kA = 16u * 8u * kTcBM;   // A bytes of a stage
  constexpr size_t kStage = tc_stage_bytes<BN>();
  uint64_t* bar = reinterpret_cast<uint64_t*>(tc_smem + kTcStages * kStage);   // [kTcStages] MMA done
  uint64_t* done_bar = bar + kTcStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done_bar + 1);

  const int p0 = blockIdx.x * kTcBM;
  const int n0 = blockIdx.y * BN;
  const int K = 9 * a.cin;
  const int nk = (K + kTcBK - 1) / kTcBK;
  const int outN2 = a.out_n * a.out_n;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"((uint32_t)tc_cols<BN>())
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int s = 0; s < kTcStages; ++s) mbar_init(bar + s, 1);
    mbar_init(done_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  // this thread's row (output node) of A
  const int p = p0 + tid;
  const bool r_ok = p < a.total;
  const int img = r_ok ? p / outN2 : 0;
  const int q = r_ok ? p - img * outN2 : 0;
  const int qy = q / a.out_n, qx = q - (q / a.out_n) * a.out_n;
  const bf16* in_img = a.in + (size_t)img * a.in_img;

  auto load_stage = [&](int s, int kt) {
    unsigned char* As = tc_smem + (size_t)s * kStage;
    unsigned char* Bs = As + kA;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int k = kt * kTcBK + c * 8;
      const bf16* src = a.in;
      bool ok = r_ok && k < K;
      if (ok) {
        const int tap = k / a.cin, ci = k - (k / a.cin) * a.cin;
        int sy, sx;
        ok = conv_src(0, a.stride, a.in_n, qy, qx, tap / 3 - 1, tap % 3 - 1, sy, sx);
        if (ok) src = in_img + ((size_t)sy * a.in_n + sx) * a.in_cs + ci;
      }
      cp_async16(As + ((size_t)c * kTcBM + tid) * 16, src, ok ? 16 : 0);
    }
    for (int u = tid; u < BN * 8; u += 128) {
      const int n = u % BN, c = u / BN;
      const int k = kt * kTcBK + c * 8;
      const bool ok = k < K;
      cp_async16(Bs + ((size_t)c * BN + n) * 16, ok ? a.w + (size_t)(n0 + n) * K + k : a.w, ok ? 16 : 0);
    }
  };

  bool fail = false;
#pragma unroll
  for (int s = 0; s < kTcStages - 1; ++s) {
    if (s < nk) load_stage(s, s);
    cp_async_commit();
  }
  constexpr uint32_t idesc = tc_idesc(BN);
  for (int kt = 0; kt < nk && !fail; ++kt) {
    const int s = kt % kTcStages;
    cp_async_wait<kTcStages - 2>();
    fence_async_smem();   // this thread's gathers, visible to the tensor core
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t as = smem_u32(tc_smem + (size_t)s * kStage), bs = as + kA;
#pragma unroll
      for (int j = 0; j < kTcBK / 16; ++j) {
        if (kt * kTcBK + j * 16 >= K) break;
        const uint64_t ad = tc_desc(as + j * 2 * (16 * kTcBM), 16 * kTcBM, 128);
        const uint64_t bd = tc_desc(bs + j * 2 * (16 * BN), 16 * BN, 128);
        tc_mma(tmem, ad, bd, idesc, (kt > 0 || j > 0) ? 1u : 0u);
      }
      tc_commit(bar + s);
    }
    // refill the stage the previous iteration's MMAs read, once they are done
    const int kn = kt + kTcStages - 1;
    if (kn < nk) {
      const int sn = kn % kTcStages;
      if (kt >= 1 && !mbar_wait(bar + sn, (uint32_t)(((kt - 1) / kTcStages) & 1))) fail = true;
      if (!fail) load_stage(sn, kn);
    }
    cp_async_commit();
    fail = __syncthreads_or(fail) != 0;
  }
  // every MMA issued (also after a failed wait) completes before the
  // accumulator is read or freed
  if (tid == 0) tc_commit(done_bar);
  if (!mbar_wait(done_bar, 0)) fail = true;
  cp_async_wait<0>();
  fail = __syncthreads_or(fail) != 0;
  tc_fence_after();

  if (!fail) {
    // epilogue: row tid of the tile from TMEM lane tid (warp w reads lanes 32w..32w+31)
    const size_t ob = (size_t)img * a.out_img + (size_t)q * a.out_cs;
    const bf16* mk = a.mask ? a.mask + (size_t)img * a.mask_img + (size_t)q * a.mask_cs : nullptr;
#pragma unroll
    for (int c0 = 0; c0 < BN; c0 += 16) {
      uint32_t r[16];
      tc_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
      tc_wait_ld();
      if (!r_ok) continue;
      float v[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const int co = n0 + c0 + e;
        v[e] = __uint_as_float(r[e]);
        if (co >= a.cout) continue;
        if (a.bias) v[e] += a.bias[co];
        if (a.accumulate) {
          v[e] += a.out_f32 ? static_cast<const float*>(a.out)[ob + co]
                            : __bfloat162float(static_cast<const bf16*>(a.out)[ob + co]);
        }
        if (a.relu) v[e] = fmaxf(v[e], 0.f);
        if (mk && !(__bfloat162float(mk[co]) > 0.f)) v[e] = 0.f;
      }
      const int cb = n0 + c0;
      if (a.out_f32) {
        float* o = static_cast<float*>(a.out) + ob;
#pragma unroll
        for (int e = 0; e < 16; ++e)
          if (cb + e < a.cout) o[cb + e] = v[e];
      } else if (cb + 16 <= a.cout) {
        // 16 channels from an even channel of a node whose channel stride and
        // view offset are multiples of 8: 16-byte aligned
        uint4 pk[2];
        __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(pk);
#pragma unroll
        for (int e = 0; e < 8; ++e) h[e] = __floats2bfloat162_rn(v[2 * e], v[2 * e + 1]);
        uint4* o = reinterpret_cast<uint4*>(static_cast<bf16*>(a.out) + ob + cb);
        o[0] = pk[0];
        o[1] = pk[1];
      } else {
        bf16* o = static_cast<bf16*>(a.out) + ob;
#pragma unroll
        for (int e = 0; e < 16; ++e)
          if (cb + e < a.cout) o[cb + e] = __float2bfloat16(v[e]);
      }
    }
  } else if (tid == 0) {
    atomicExch(err, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)tc_cols<BN>())
                 : "memory");
  }
}

// ---------------------------------------------------------------------------
// k_conv_row_tc: the same forward convolution with the input staged once per
// tile.  A tile is R output rows (qy0..qy0+R-1) x 128 consecutive output
// nodes (qx0..qx0+127); the Hr = S (R - 1) + 3 input rows it reads are
// staged in shared memory as a halo of 16-byte units, K chunk (8 channels)
// outermost: unit (c, h, i) at ((c * Hr + h) * W + i) * 16 bytes, i the node
// of the halo row (stride 1: input x = qx0 - 1 + i, W = 130; stride 2: the
// odd columns 2 qx0 - 1 + 2 i for i < 129, then the even columns
// 2 qx0 + 2 (i - 129), W = 257).  The A operand of output row r and tap
// (dy, dx) is the halo itself from row h = S r + dy + 1 and the node where
// the tap's column starts (stride 1: i = m + dx + 1; stride 2: odd i = m
// (dx = -1) or m + 1 (dx = 1), even i = 129 + m): a descriptor with an offset
// start address, rows 16 bytes apart, 8-row groups 128 bytes apart, the two
// K chunks of an MMA Hr W x 16 bytes apart -- every input node is fetched once
// per tile instead of once per tap and output row.  Output row r accumulates
// in TMEM columns [r BN, (r + 1) BN).
// The channels are taken in groups of G (a multiple of 16 dividing cin): a
// unit of work is (tile, group); its halo and the group's weights of all 9
// taps ([tap][chunk][BN rows] of 16-byte units) fill one of two shared-memory
// slots while the tensor core works on the other (with a single group the
// weights stay in their slots).  The CTAs are persistent over the tiles
// (tile = blockIdx.x + k gridDim.x); a tile's accumulators are read by the
// epilogue after its last group.  One thread issues the MMAs and waits on the
// mbarriers; the others wait at the CTA barrier.
template <int S>
__host__ __device__ constexpr int row_tc_w() { return S == 1 ? 130 : 257; }
// Output rows per tile: 128 accumulator columns' worth, at least two -- the
// MMAs of different rows are independent, and they are issued interleaved so
// that the tensor core overlaps them (a chain of small MMAs on one
// accumulator waits on each other).
__host__ __device__ constexpr int row_tc_rows(int BN) { return BN >= 64 ? 2 : 128 / BN; }
template <int BN, int S>
__host__ __device__ constexpr size_t row_tc_slot(int G) {
  return (size_t)G * 2 * ((size_t)(S * (row_tc_rows(BN) - 1) + 3) * row_tc_w<S>() + 9 * BN);
}
template <int BN, int S>
__host__ __device__ constexpr size_t row_tc_smem(int G) {
  return 2 * row_tc_slot<BN, S>(G) + 128;
}
template <int BN>
__host__ __device__ constexpr int row_tc_cols() {
  return BN * row_tc_rows(BN) < 32 ? 32 : BN * row_tc_rows(BN);
}

template <int BN, int S>
__global__ void __launch_bounds__(128) k_conv_row_tc(ConvArgs a, int G, int* err) {
  extern __shared__ __align__(1024) unsigned char rt_smem[];
  constexpr int W = row_tc_w<S>();
  constexpr int R = row_tc_rows(BN);
  constexpr int Hr = S * (R - 1) + 3;
  constexpr uint32_t kCols = (uint32_t)row_tc_cols<BN>();
  const int tid = threadIdx.x, warp = tid >> 5;
  const size_t slot_bytes = row_tc_slot<BN, S>(G);
  const size_t halo_bytes = (size_t)G * 2 * Hr * W;
  uint64_t* bar = reinterpret_cast<uint64_t*>(rt_smem + 2 * slot_bytes);   // [2] MMAs of a slot done
  uint64_t* done_bar = bar + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done_bar + 1);
  __shared__ int s_fail;

  const int segs = (a.out_n + kTcBM - 1) / kTcBM;
  const int rgs = (a.out_n + R - 1) / R;   // row groups per image
  const int images = a.total / (a.out_n * a.out_n);
  const int tiles = images * rgs * segs;
  const int ng = a.cin / G, cpg = G / 8;
  const int n0 = blockIdx.y * BN;
  const int K = 9 * a.cin;
  const int my_tiles = (int)blockIdx.x < tiles ? (tiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int U = my_tiles * ng;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_init(bar + 1, 1);
    mbar_init(done_bar, 1);
    s_fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  auto tile_of_unit = [&](int u, int& img, int& qy0, int& qx0, int& g) {
    const int t = (int)blockIdx.x + (u / ng) * (int)gridDim.x;
    g = u - (u / ng) * ng;
    img = t / (rgs * segs);
    const int r = t - img * (rgs * segs);
    const int rg = r / segs;
    qy0 = rg * R;
    qx0 = (r - rg * segs) * kTcBM;
  };
  auto load_unit = [&](int u, int slot) {
    int img, qy0, qx0, g;
    tile_of_unit(u, img, qy0, qx0, g);
    unsigned char* H = rt_smem + (size_t)slot * slot_bytes;
    const bf16* in_img = a.in + (size_t)img * a.in_img + g * G;
    // halo: (chunk, row) lines of W units
    for (int line = warp; line < cpg * Hr; line += 4) {
      const int c = line / Hr, h = line - (line / Hr) * Hr;
      const int y = S * qy0 + h - 1;
      const bool yok = y >= 0 && y < a.in_n;
      const bf16* row = in_img + (size_t)(yok ? y : 0) * a.in_n * a.in_cs + 8 * c;
      unsigned char* dst = H + (size_t)line * W * 16;
      for (int i = tid & 31; i < W; i += 32) {
        const int x = (S == 1) ? qx0 - 1 + i : (i < 129 ? 2 * qx0 - 1 + 2 * i : 2 * qx0 + 2 * (i - 129));
        const bool ok = yok && x >= 0 && x < a.in_n;
        cp_async16(dst + (size_t)i * 16, ok ? row + (size_t)x * a.in_cs : a.in, ok ? 16 : 0);
      }
    }
    // weights of the group (a single group: already in the slot after its first use)
    if (ng > 1 || u < 2) {
      unsigned char* Wt = H + halo_bytes;
      const int nw = 9 * cpg * BN;
      for (int e = tid; e < nw; e += 128) {
        const int n = e % BN, tc = e / BN, tap = tc / cpg, c = tc - tap * cpg;
        cp_async16(Wt + (size_t)e * 16, a.w + (size_t)(n0 + n) * K + tap * a.cin + g * G + 8 * c, 16);
      }
    }
  };

  constexpr uint32_t idesc = tc_idesc(BN);
  if (U > 0) load_unit(0, 0);
  cp_async_commit();
  for (int u = 0; u < U; ++u) {
    const int slot = u & 1;
    // the other slot's MMAs (unit u - 1) done before it is refilled with unit u + 1
    if (u + 1 < U) {
      if (u >= 1 && tid == 0 && !mbar_wait(bar + ((u + 1) & 1), (uint32_t)(((u - 1) >> 1) & 1))) s_fail = 1;
      __syncthreads();
      if (s_fail) break;
      load_unit(u + 1, (u + 1) & 1);
    }
    cp_async_commit();
    cp_async_wait<1>();   // unit u's copies (this thread's)
    fence_async_smem();
    __syncthreads();
    int img, qy0, qx0, g;
    tile_of_unit(u, img, qy0, qx0, g);
    if (tid == 0) {
      tc_fence_after();
      const uint32_t hb = smem_u32(rt_smem + (size_t)slot * slot_bytes), wb = hb + (uint32_t)halo_bytes;
      const uint32_t lbo_a = (uint32_t)Hr * W * 16u;
      const int rr = min(R, a.out_n - qy0);
      for (int tap = 0; tap < 9; ++tap) {
        const int dy = tap / 3 - 1, dx = tap % 3 - 1;
        const int i0 = (S == 1) ? dx + 1 : (dx == 0 ? 129 : (dx < 0 ? 0 : 1));
        for (int j = 0; j < cpg / 2; ++j) {
          const uint64_t bd = tc_desc(wb + (uint32_t)((tap * cpg + 2 * j) * BN * 16), BN * 16, 128);
          const uint32_t acc = (g > 0 || tap > 0 || j > 0) ? 1u : 0u;
          for (int r = 0; r < rr; ++r) {
            const int h = S * r + dy + 1;
            const uint64_t ad = tc_desc(hb + (uint32_t)(((2 * j * Hr + h) * W + i0) * 16), lbo_a, 128);
            tc_mma(tmem + (uint32_t)(r * BN), ad, bd, idesc, acc);
          }
        }
      }
      tc_commit(bar + slot);
    }
    if (g == ng - 1) {
      // the tile's accumulators are complete once this unit's MMAs are
      if (tid == 0 && !mbar_wait(bar + slot, (uint32_t)((u >> 1) & 1))) s_fail = 1;
      __syncthreads();
      if (s_fail) break;
      tc_fence_after();
      const int qx = qx0 + tid;
      const bool xok = qx < a.out_n;
      for (int r = 0; r < R; ++r) {
        if (qy0 + r >= a.out_n) break;
        const size_t q = (size_t)(qy0 + r) * a.out_n + qx;
        const size_t ob = (size_t)img * a.out_img + q * a.out_cs;
        const bf16* mk = a.mask ? a.mask + (size_t)img * a.mask_img + q * a.mask_cs : nullptr;
#pragma unroll
        for (int c0 = 0; c0 < BN; c0 += 16) {
          uint32_t rv[16];
          tc_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(r * BN + c0), rv);
          tc_wait_ld();
          if (!xok) continue;
          float v[16];
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            const int co = n0 + c0 + e;
            v[e] = __uint_as_float(rv[e]);
            if (co >= a.cout) continue;
            if (a.bias) v[e] += __ldg(a.bias + co);
            if (a.accumulate) {
              v[e] += a.out_f32 ? static_cast<const float*>(a.out)[ob + co]
                                : __bfloat162float(static_cast<const bf16*>(a.out)[ob + co]);
            }
            if (a.relu) v[e] = fmaxf(v[e], 0.f);
            if (mk && !(__bfloat162float(mk[co]) > 0.f)) v[e] = 0.f;
          }
          const int cb = n0 + c0;
          if (a.out_f32) {
            float* o = static_cast<float*>(a.out) + ob;
#pragma unroll
            for (int e = 0; e < 16; ++e)
              if (cb + e < a.cout) o[cb + e] = v[e];
          } else if (cb + 16 <= a.cout) {
            uint4 pk[2];
            __nv_bfloat162* hh = reinterpret_cast<__nv_bfloat162*>(pk);
#pragma unroll
            for (int e = 0; e < 8; ++e) hh[e] = __floats2bfloat162_rn(v[2 * e], v[2 * e + 1]);
            uint4* o = reinterpret_cast<uint4*>(static_cast<bf16*>(a.out) + ob + cb);
            o[0] = pk[0];
            o[1] = pk[1];
          } else {
            bf16* o = static_cast<bf16*>(a.out) + ob;
#pragma unroll
            for (int e = 0; e < 16; ++e)
              if (cb + e < a.cout) o[cb + e] = __float2bfloat16(v[e]);
          }
        }
      }
      // the next tile's first MMAs overwrite the accumulators: after every read
      tc_fence_before();
      __syncthreads();
    }
  }
  if (s_fail && tid == 0) atomicExch(err, 1);
  // every MMA issued completes before the accumulators are freed
  if (tid == 0) {
    tc_commit(done_bar);
    mbar_wait(done_bar, 0);
  }
  cp_async_wait<0>();
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
  }
}

// ---------------------------------------------------------------------------
// k_conv_row_tma: the stride-1 row-tile convolution of k_conv_row_tc with its
// operands brought by the Tensor Memory Accelerator and its work split over
// warps.  Warp 4 (one elected thread) drives the tile loop: per unit it posts
// the expected bytes on the slot's mbarrier and issues the tensor copies --
// per 8-channel chunk one box (8 channels x 130 nodes x Hr rows x 1 image) of
// the NHWC input, out-of-grid nodes filled with zeros by the copy engine,
// landing as the halo's (row, node) units; per (tap, chunk) one box (8 K
// elements x BN weight rows) -- waits for the bytes, issues the MMAs and
// commits.  Warps 0-3 read the accumulators of a finished tile (warp w: TMEM
// lanes 32w..32w+31) and store the outputs.  Two accumulator sets in TMEM let
// the epilogue of one tile overlap the MMAs of the next; two operand slots
// let the copies of one unit overlap the MMAs of another.  No copy uses
// cluster multicast.
constexpr int kRowTmaThreads = 160;
__host__ __device__ constexpr uint32_t row_tma_chunk(int BN) {
  return ((uint32_t)(row_tc_rows(BN) + 2) * 130u * 16u + 127u) & ~127u;
}
__host__ __device__ constexpr uint32_t row_tma_slot(int BN, int G) {
  return ((uint32_t)(G / 8) * row_tma_chunk(BN) + 9u * (uint32_t)(G / 8) * (uint32_t)BN * 16u + 1023u) & ~1023u;
}
__host__ __device__ constexpr size_t row_tma_smem(int BN, int G) {
  return 2 * (size_t)row_tma_slot(BN, G) + 1024 + 128;
}
template <int BN>
__host__ __device__ constexpr int row_tma_cols() {
  return 2 * row_tc_rows(BN) * BN < 32 ? 32 : 2 * row_tc_rows(BN) * BN;
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int c0, int c1, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
      : "memory");
}

template <int BN>
__global__ void __launch_bounds__(kRowTmaThreads) k_conv_row_tma(ConvArgs a, int G, int* err,
                                                                 const __grid_constant__ CUtensorMap tin,
                                                                 const __grid_constant__ CUtensorMap tw) {
  extern __shared__ __align__(1024) unsigned char tm_raw[];
  constexpr int W = 130;
  constexpr int R = row_tc_rows(BN);
  constexpr int Hr = R + 2;
  constexpr uint32_t kCols = (uint32_t)row_tma_cols<BN>();
  constexpr uint32_t CS = row_tma_chunk(BN);
  unsigned char* sm = tm_raw + ((1024u - (smem_u32(tm_raw) & 1023u)) & 1023u);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int cpg = G / 8;
  const uint32_t halo_bytes = (uint32_t)cpg * CS;
  const uint32_t w_bytes = 9u * (uint32_t)cpg * BN * 16u;
  const uint32_t slot_bytes = row_tma_slot(BN, G);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + 2 * (size_t)slot_bytes);   // [2] bytes of a slot landed
  uint64_t* mma_bar = full + 2;      // [2] MMAs reading a slot done
  uint64_t* acc_full = full + 4;     // [2] accumulator set complete
  uint64_t* acc_empty = full + 6;    // [2] accumulator set read by the epilogue
  uint64_t* done_bar = full + 8;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(full + 9);
  volatile int* fail = reinterpret_cast<volatile int*>(full + 10);

  const int segs = (a.out_n + kTcBM - 1) / kTcBM;
  const int rgs = (a.out_n + R - 1) / R;
  const int images = a.total / (a.out_n * a.out_n);
  const int tiles = images * rgs * segs;
  const int ng = a.cin / G;
  const int n0 = blockIdx.y * BN;
  const int my_tiles = (int)blockIdx.x < tiles ? (tiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int U = my_tiles * ng;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int k = 0; k < 6; ++k) mbar_init(full + k, 1);
    mbar_init(acc_empty, 128);
    mbar_init(acc_empty + 1, 128);
    mbar_init(done_bar, 1);
    *fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  auto tile_at = [&](int ti, int& img, int& qy0, int& qx0) {
    const int t = (int)blockIdx.x + ti * (int)gridDim.x;
    img = t / (rgs * segs);
    const int r = t - img * (rgs * segs);
    const int rg = r / segs;
    qy0 = rg * R;
    qx0 = (r - rg * segs) * kTcBM;
  };

  if (warp == 4) {
    if ((tid & 31) == 0) {
      int posts[2] = {0, 0}, landed[2] = {0, 0};
      auto issue_loads = [&](int u, int slot) {
        int img, qy0, qx0;
        tile_at(u / ng, img, qy0, qx0);
        const int g = u % ng;
        const bool with_w = ng > 1 || u < 2;
        ++posts[slot];
        mbar_expect_tx(full + slot, (uint32_t)cpg * (Hr * W * 16u) + (with_w ? w_bytes : 0u));
        const uint32_t hb = smem_u32(sm + (size_t)slot * slot_bytes);
        for (int c = 0; c < cpg; ++c)
          tma_load_4d(hb + (uint32_t)c * CS, &tin, g * G + 8 * c, qx0 - 1, qy0 - 1, img, full + slot);
        if (with_w) {
          const uint32_t wb = hb + halo_bytes;
          for (int tap = 0; tap < 9; ++tap)
            for (int c = 0; c < cpg; ++c)
              tma_load_2d(wb + (uint32_t)((tap * cpg + c) * BN * 16), &tw, tap * a.cin + g * G + 8 * c, n0, full + slot);
        }
      };
      constexpr uint32_t idesc = tc_idesc(BN);
      if (U > 0) issue_loads(0, 0);
      for (int u = 0; u < U && !*fail; ++u) {
        const int slot = u & 1, ti = u / ng, g = u % ng, as = ti & 1;
        if (u + 1 < U) {
          if (u >= 1 && !mbar_wait(mma_bar + ((u + 1) & 1), (uint32_t)(((u - 1) >> 1) & 1))) { *fail = 1; break; }
          issue_loads(u + 1, (u + 1) & 1);
        }
        if (!mbar_wait(full + slot, (uint32_t)((u >> 1) & 1))) { *fail = 1; break; }
        ++landed[slot];
        // the accumulator set was read by the epilogue of tile ti - 2
        if (g == 0 && ti >= 2 && !mbar_wait(acc_empty + as, (uint32_t)(((ti - 2) >> 1) & 1))) { *fail = 1; break; }
        tc_fence_after();
        int img, qy0, qx0;
        tile_at(ti, img, qy0, qx0);
        const uint32_t hb = smem_u32(sm + (size_t)slot * slot_bytes), wb = hb + halo_bytes;
        const uint32_t acc_base = tmem + (uint32_t)(as * R * BN);
        const int rr = min(R, a.out_n - qy0);
        for (int tap = 0; tap < 9; ++tap) {
          const int dy = tap / 3 - 1, dx = tap % 3 - 1;
          for (int j = 0; j < cpg / 2; ++j) {
            const uint64_t bd = tc_desc(wb + (uint32_t)((tap * cpg + 2 * j) * BN * 16), BN * 16, 128);
            const uint32_t accf = (g > 0 || tap > 0 || j > 0) ? 1u : 0u;
            const uint64_t ad0 = tc_desc(hb + (uint32_t)(2 * j) * CS + (uint32_t)(((dy + 1) * W + dx + 1) * 16), CS, 128);
            for (int r = 0; r < rr; ++r)   // the start address field advances by W units per row
              tc_mma(acc_base + (uint32_t)(r * BN), ad0 + (uint64_t)(r * W), bd, idesc, accf);
          }
        }
        tc_commit(mma_bar + slot);
        if (g == ng - 1) tc_commit(acc_full + as);
      }
      // every copy posted and every MMA issued complete before the block ends
      for (int k = 0; k < 2; ++k)
        if (posts[k] > landed[k]) mbar_wait(full + k, (uint32_t)((posts[k] - 1) & 1));
      tc_commit(done_bar);
      mbar_wait(done_bar, 0);
    }
  } else {
    // epilogue warps: tile after tile, from the accumulator set it was computed in
    for (int ti = 0; ti < my_tiles; ++ti) {
      const int as = ti & 1;
      if (!mbar_wait(acc_full + as, (uint32_t)((ti >> 1) & 1))) {
        *fail = 1;
        break;
      }
      if (*fail) break;
      tc_fence_after();
      int img, qy0, qx0;
      tile_at(ti, img, qy0, qx0);
      const int qx = qx0 + tid;
      const bool xok = qx < a.out_n;
      for (int r = 0; r < R; ++r) {
        if (qy0 + r >= a.out_n) break;
        const size_t q = (size_t)(qy0 + r) * a.out_n + qx;
        const size_t ob = (size_t)img * a.out_img + q * a.out_cs;
        const bf16* mk = a.mask ? a.mask + (size_t)img * a.mask_img + q * a.mask_cs : nullptr;
#pragma unroll
        for (int c0 = 0; c0 < BN; c0 += 16) {
          uint32_t rv[16];
          tc_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((as * R + r) * BN + c0), rv);
          tc_wait_ld();
          if (!xok) continue;
          float v[16];
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            const int co = n0 + c0 + e;
            v[e] = __uint_as_float(rv[e]);
            if (co >= a.cout) continue;
            if (a.bias) v[e] += __ldg(a.bias + co);
            if (a.accumulate) {
              v[e] += a.out_f32 ? static_cast<const float*>(a.out)[ob + co]
                                : __bfloat162float(static_cast<const bf16*>(a.out)[ob + co]);
            }
            if (a.relu) v[e] = fmaxf(v[e], 0.f);
            if (mk && !(__bfloat162float(mk[co]) > 0.f)) v[e] = 0.f;
          }
          const int cb = n0 + c0;
          if (a.out_f32) {
            float* o = static_cast<float*>(a.out) + ob;
#pragma unroll
            for (int e = 0; e < 16; ++e)
              if (cb + e < a.cout) o[cb + e] = v[e];
          } else if (cb + 16 <= a.cout) {
            uint4 pk[2];
            __nv_bfloat162* hh = reinterpret_cast<__nv_bfloat162*>(pk);
#pragma unroll
            for (int e = 0; e < 8; ++e) hh[e] = __floats2bfloat162_rn(v[2 * e], v[2 * e + 1]);
            uint4* o = reinterpret_cast<uint4*>(static_cast<bf16*>(a.out) + ob + cb);
            o[0] = pk[0];
            o[1] = pk[1];
          } else {
            bf16* o = static_cast<bf16*>(a.out) + ob;
#pragma unroll
            for (int e = 0; e < 16; ++e)
              if (cb + e < a.cout) o[cb + e] = __float2bfloat16(v[e]);
          }
        }
      }
      tc_fence_before();
      mbar_arrive(acc_empty + as);
    }
  }
  __syncthreads();
  if (tid == 0 && *fail) atomicExch(err, 1);
  tc_fence_after();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
  }
}

}  // namespace unet
}  // namespace msg
