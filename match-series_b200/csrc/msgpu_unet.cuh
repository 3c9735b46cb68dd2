// msgpu_unet.cuh -- kernels of the learned warm start: a U-Net on 2^l+1
// node grids that maps the normalised reference/template pair of a frame to
// a coarse displacement, trained and run on the GPU.
//
// Tensors are NHWC bf16 "views": image stride, nodes per side, elements per
// node (channel stride) and a channel offset in the base pointer, so the
// decoder's concatenations [skip | upsampled] are channel slices of one
// buffer and no copy is made.  Channel counts are padded to multiples of 16.
//
// k_conv: one 3x3 convolution as an implicit GEMM on the tensor pipe
// (mma.sync m16n8k16, bf16 operands, fp32 accumulation).  A block computes
// 128 output nodes x BN output channels; the reduction runs over
// (tap, input channel) in stages of 32, staged in shared memory by a
// three-stage cp.async pipeline with zero fill for taps outside the grid,
// fragments loaded by ldmatrix.  mode 0 reads input
// node stride*q + d (forward), mode 1 reads (q - d)/stride when that is a
// node (the data gradient of a forward convolution, with the weights
// transposed).  The epilogue adds the bias, accumulates into the output,
// applies ReLU and a ReLU mask as asked.
//
// k_wgrad: weight gradient dW[co][(tap, ci)] = sum over nodes of
// dY[node][co] * X[src(node, tap)][ci] and the bias gradient, the node sum
// split into chunks; each block writes its chunk's partial, k_wgrad_reduce
// and k_bgrad_reduce add the partials in chunk order (deterministic
// training).
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace msg {
namespace unet {

typedef __nv_bfloat16 bf16;

constexpr int kThreads = 128;
constexpr int kBK = 32;        // reduction elements per stage
constexpr int kSA = kBK + 8;   // shared-memory row stride (bf16): conflict-free fragment loads

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// source node of output node (qy, qx) under tap (dy, dx); false when there is none
__device__ __forceinline__ bool conv_src(int mode, int stride, int n_in, int qy, int qx, int dy, int dx, int& sy,
                                         int& sx) {
  if (mode == 0) {
    sy = stride * qy + dy;
    sx = stride * qx + dx;
  } else {
    const int ty = qy - dy, tx = qx - dx;
    if (stride == 2) {
      if ((ty | tx) & 1) return false;
      sy = ty >> 1;
      sx = tx >> 1;
    } else {
      sy = ty;
      sx = tx;
    }
  }
  return sy >= 0 && sy < n_in && sx >= 0 && sx < n_in;
}

struct ConvArgs {
  const bf16* in;        // input view: image 0, first channel read
  size_t in_img;         // elements between images
  int in_n, in_cs, cin;  // nodes per side, elements per node, channels read (multiple of 16)
  const bf16* w;         // [rows][9 * cin], (tap, channel) contiguous
  const float* bias;     // nullable, [cout]
  void* out;             // output view (bf16, or float with out_f32)
  size_t out_img;
  int out_n, out_cs, cout;   // channels stored
  int out_f32;
  int mode, stride, relu, accumulate;
  const bf16* mask;      // nullable: output zeroed where mask <= 0
  size_t mask_img;
  int mask_cs;
  int total;             // images * out_n^2
};

__device__ __forceinline__ void ldsm_x4(uint32_t* r, const void* smem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(s));
}
__device__ __forceinline__ void ldsm_x4_trans(uint32_t* r, const void* smem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(s));
}

constexpr int kConvBM = 128;   // output nodes per conv block (32 per warp)
constexpr int kStages = 3;

// Block: 128 output nodes x BN channels, 4 warps of 32 nodes each (two m16
// tiles sharing every B fragment); fragments by ldmatrix from rows of 80
// bytes (conflict-free); three cp.async stages.
template <int BN>
__global__ void __launch_bounds__(kThreads) k_conv(ConvArgs a) {
  extern __shared__ __align__(16) unsigned char conv_smem[];
  bf16 (*As)[kConvBM][kSA] = reinterpret_cast<bf16 (*)[kConvBM][kSA]>(conv_smem);
  bf16 (*Bs)[BN][kSA] = reinterpret_cast<bf16 (*)[BN][kSA]>(conv_smem + sizeof(bf16) * kStages * kConvBM * kSA);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int p0 = blockIdx.x * kConvBM;
  const int n0 = blockIdx.y * BN;
  const int K = 9 * a.cin;
  const int nk = (K + kBK - 1) / kBK;
  const int outN2 = a.out_n * a.out_n;
  // the four rows (nodes) this thread loads: row = tid / 4 + 32 i
  int r_img[4], r_qy[4], r_qx[4];
  bool r_ok[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int p = p0 + (tid >> 2) + 32 * i;
    r_ok[i] = p < a.total;
    const int img = r_ok[i] ? p / outN2 : 0;
    const int q = r_ok[i] ? p - img * outN2 : 0;
    r_img[i] = img;
    r_qy[i] = q / a.out_n;
    r_qx[i] = q - r_qy[i] * a.out_n;
  }
  const int g = tid & 3;
  auto load_stage = [&](int s, int kt) {
    const int k = kt * kBK + g * 8;
    const bool kin = k < K;
    int tap = 0, ci = 0;
    if (kin) {
      tap = k / a.cin;
      ci = k - tap * a.cin;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const bf16* src = a.in;
      bool ok = r_ok[i] && kin;
      if (ok) {
        int sy, sx;
        ok = conv_src(a.mode, a.stride, a.in_n, r_qy[i], r_qx[i], tap / 3 - 1, tap % 3 - 1, sy, sx);
        if (ok) src = a.in + (size_t)r_img[i] * a.in_img + ((size_t)sy * a.in_n + sx) * a.in_cs + ci;
      }
      cp_async16(&As[s][(tid >> 2) + 32 * i][g * 8], src, ok ? 16 : 0);
    }
    for (int idx = tid; idx < BN * 4; idx += kThreads) {
      const int row = idx >> 2, gg = idx & 3;
      const int kk = kt * kBK + gg * 8;
      const bool ok = kk < K;
      cp_async16(&Bs[s][row][gg * 8], ok ? a.w + (size_t)(n0 + row) * K + kk : a.w, ok ? 16 : 0);
    }
  };
  float acc[2][BN / 8][4];
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int j = 0; j < BN / 8; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[m][j][e] = 0.f;
#pragma unroll
  for (int s = 0; s < kStages - 1; ++s) {
    if (s < nk) load_stage(s, s);
    cp_async_commit();
  }
  // ldmatrix lane addresses: A rows r0 + lane % 16, column + 8 (lane / 16);
  // B rows n + lane % 8 + 8 (lane / 16), column + 8 ((lane / 8) % 2)
  const int a_row = warp * 32 + (lane & 15), a_col = 8 * (lane >> 4);
  const int b_row = (lane & 7) + 8 * (lane >> 4), b_col = 8 * ((lane >> 3) & 1);
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<kStages - 2>();
    __syncthreads();
    {
      const int kn = kt + kStages - 1;
      if (kn < nk) load_stage(kn % kStages, kn);
      cp_async_commit();
    }
    const int s = kt % kStages;
#pragma unroll
    for (int kk = 0; kk < kBK; kk += 16) {
      uint32_t af[2][4];
      ldsm_x4(af[0], &As[s][a_row][kk + a_col]);
      ldsm_x4(af[1], &As[s][a_row + 16][kk + a_col]);
#pragma unroll
      for (int j = 0; j < BN / 8; j += 2) {
        uint32_t bf[4];
        ldsm_x4(bf, &Bs[s][j * 8 + b_row][kk + b_col]);
#pragma unroll
        for (int m = 0; m < 2; ++m) {
          mma_bf16(acc[m][j], af[m], bf[0], bf[1]);
          mma_bf16(acc[m][j + 1], af[m], bf[2], bf[3]);
        }
      }
    }
  }
  cp_async_wait<0>();
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int p = p0 + warp * 32 + 16 * m + (lane >> 2) + 8 * h;
      if (p >= a.total) continue;
      const int img = p / outN2, q = p - img * outN2;
      const size_t ob = (size_t)img * a.out_img + (size_t)q * a.out_cs;
      const bf16* mk = a.mask ? a.mask + (size_t)img * a.mask_img + (size_t)q * a.mask_cs : nullptr;
#pragma unroll
      for (int j = 0; j < BN / 8; ++j) {
        const int co = n0 + j * 8 + 2 * (lane & 3);
        float v[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          v[e] = acc[m][j][2 * h + e];
          if (co + e >= a.cout) continue;
          if (a.bias) v[e] += a.bias[co + e];
          if (a.accumulate) v[e] += __bfloat162float(static_cast<const bf16*>(a.out)[ob + co + e]);
          if (a.relu) v[e] = fmaxf(v[e], 0.f);
          if (mk && !(__bfloat162float(mk[co + e]) > 0.f)) v[e] = 0.f;
        }
        if (a.out_f32) {
          float* o = static_cast<float*>(a.out) + ob;
          if (co < a.cout) o[co] = v[0];
          if (co + 1 < a.cout) o[co + 1] = v[1];
        } else if (co + 1 < a.cout) {
          // co even, channel stride and view offsets multiples of 8: 4-byte aligned
          *reinterpret_cast<__nv_bfloat162*>(static_cast<bf16*>(a.out) + ob + co) = __floats2bfloat162_rn(v[0], v[1]);
        } else if (co < a.cout) {
          static_cast<bf16*>(a.out)[ob + co] = __float2bfloat16(v[0]);
        }
      }
    }
}

template <int BN>
constexpr size_t conv_smem_bytes() {
  return sizeof(bf16) * kStages * (kConvBM + BN) * kSA;
}

// Stride-1 convolution (forward, or the data gradient with transposed
// weights) of CIN = 16 or 32 input channels from a halo tile: a block
// computes (4 MT) x 16 output nodes of one image (each warp MT rows of 16,
// one m16 tile per row) x BN channels.  The (4MT+2) x (16+2) input nodes and all 9
// taps' weights are staged once in shared memory; every tap's A fragment is
// read by ldmatrix straight from the halo rows (consecutive nodes of a row,
// conflict-free), so each input node is fetched once instead of once per
// tap.  The mma sequence over (tap, channel) is the one k_conv issues, so
// both give the same results.
constexpr int kHaloX = 16;
template <int CIN>
__host__ __device__ constexpr int halo_stride() { return CIN + 8; }
template <int BN, int CIN, int MT>
constexpr size_t conv_halo_smem_bytes() {
  return sizeof(bf16) * ((size_t)(4 * MT + 2) * (kHaloX + 2) * halo_stride<CIN>() + (size_t)9 * BN * halo_stride<CIN>());
}

template <int BN, int CIN, int MT>
__global__ void __launch_bounds__(kThreads) k_conv_halo(ConvArgs a) {
  constexpr int HS = halo_stride<CIN>();
  constexpr int kHaloY = 4 * MT;
  constexpr int HW = kHaloX + 2, HH = kHaloY + 2;
  extern __shared__ __align__(16) unsigned char halo_smem[];
  bf16* H = reinterpret_cast<bf16*>(halo_smem);   // [HH][HW][HS]
  bf16* W = H + (size_t)HH * HW * HS;             // [9][BN][HS]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tiles_x = (a.out_n + kHaloX - 1) / kHaloX, tiles_y = (a.out_n + kHaloY - 1) / kHaloY;
  const int img = blockIdx.x / (tiles_x * tiles_y);
  const int trest = blockIdx.x - img * tiles_x * tiles_y;
  const int ty0 = (trest / tiles_x) * kHaloY, tx0 = (trest % tiles_x) * kHaloX;
  const int n0 = blockIdx.y * BN;
  const int sgn = a.mode == 0 ? 1 : -1;   // mode 0 reads q + d, mode 1 reads q - d
  const bf16* in = a.in + (size_t)img * a.in_img;
  // halo nodes (ty0 - 1 .. ty0 + 8, tx0 - 1 .. tx0 + 16), CIN / 8 vectors each, zero outside the grid
  for (int idx = tid; idx < HH * HW * (CIN / 8); idx += kThreads) {
    const int v = idx % (CIN / 8), node = idx / (CIN / 8);
    const int hy = node / HW, hx = node - hy * HW;
    const int y = ty0 - 1 + hy, x = tx0 - 1 + hx;
    const bool ok = y >= 0 && y < a.in_n && x >= 0 && x < a.in_n;
    cp_async16(H + (size_t)node * HS + 8 * v, ok ? in + ((size_t)y * a.in_n + x) * a.in_cs + 8 * v : a.in,
               ok ? 16 : 0);
  }
  for (int idx = tid; idx < 9 * BN * (CIN / 8); idx += kThreads) {
    const int v = idx % (CIN / 8), r = idx / (CIN / 8);
    const int tap = r / BN, co = r - tap * BN;
    cp_async16(W + (size_t)r * HS + 8 * v, a.w + (size_t)(n0 + co) * 9 * CIN + tap * CIN + 8 * v, 16);
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  float acc[MT][BN / 8][4];
#pragma unroll
  for (int m = 0; m < MT; ++m)
#pragma unroll
    for (int j = 0; j < BN / 8; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[m][j][e] = 0.f;
  const int a_x = lane & 15, a_col = 8 * (lane >> 4);
  const int b_row = (lane & 7) + 8 * (lane >> 4), b_col = 8 * ((lane >> 3) & 1);
#pragma unroll 1
  for (int tap = 0; tap < 9; ++tap) {
    const int dy = sgn * (tap / 3 - 1), dx = sgn * (tap % 3 - 1);
#pragma unroll
    for (int kk = 0; kk < CIN; kk += 16) {
      uint32_t af[MT][4];
#pragma unroll
      for (int m = 0; m < MT; ++m) {
        const int hy = MT * warp + m + 1 + dy, hx = a_x + 1 + dx;
        ldsm_x4(af[m], H + ((size_t)hy * HW + hx) * HS + kk + a_col);
      }
#pragma unroll
      for (int j = 0; j < BN / 8; j += 2) {
        uint32_t bf[4];
        ldsm_x4(bf, W + ((size_t)tap * BN + j * 8 + b_row) * HS + kk + b_col);
#pragma unroll
        for (int m = 0; m < MT; ++m) {
          mma_bf16(acc[m][j], af[m], bf[0], bf[1]);
          mma_bf16(acc[m][j + 1], af[m], bf[2], bf[3]);
        }
      }
    }
  }
  const int outN2 = a.out_n * a.out_n;
  (void)outN2;
#pragma unroll
  for (int m = 0; m < MT; ++m)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int oy = ty0 + MT * warp + m, ox = tx0 + (lane >> 2) + 8 * h;
      if (oy >= a.out_n || ox >= a.out_n) continue;
      const int q = oy * a.out_n + ox;
      const size_t ob = (size_t)img * a.out_img + (size_t)q * a.out_cs;
      const bf16* mk = a.mask ? a.mask + (size_t)img * a.mask_img + (size_t)q * a.mask_cs : nullptr;
#pragma unroll
      for (int j = 0; j < BN / 8; ++j) {
        const int co = n0 + j * 8 + 2 * (lane & 3);
        float v[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          v[e] = acc[m][j][2 * h + e];
          if (co + e >= a.cout) continue;
          if (a.bias) v[e] += a.bias[co + e];
          if (a.accumulate) v[e] += __bfloat162float(static_cast<const bf16*>(a.out)[ob + co + e]);
          if (a.relu) v[e] = fmaxf(v[e], 0.f);
          if (mk && !(__bfloat162float(mk[co + e]) > 0.f)) v[e] = 0.f;
        }
        if (a.out_f32) {
          float* o = static_cast<float*>(a.out) + ob;
          if (co < a.cout) o[co] = v[0];
          if (co + 1 < a.cout) o[co + 1] = v[1];
        } else if (co + 1 < a.cout) {
          *reinterpret_cast<__nv_bfloat162*>(static_cast<bf16*>(a.out) + ob + co) = __floats2bfloat162_rn(v[0], v[1]);
        } else if (co < a.cout) {
          static_cast<bf16*>(a.out)[ob + co] = __float2bfloat16(v[0]);
        }
      }
    }
}

struct WgradArgs {
  const bf16* in;        // forward input view
  size_t in_img;
  int in_n, in_cs, cin;  // channels read (multiple of 16)
  const bf16* dy;        // gradient at the forward output (pre-activation)
  size_t dy_img;
  int dy_n, dy_cs, cout_pad;
  int stride;
  float* part;           // [chunks][cout_pad][9 * cin]
  float* bpart;          // [chunks][cout_pad]: node sums of dy (the bias gradient)
  int total;             // images * dy_n^2
  int chunk;             // nodes per block (multiple of kBK)
};

// GEMM dW^T[co][k] over node chunks: rows = output channels (BM per block),
// columns = 64 reduction indices (tap, ci), inner dimension = nodes.  Both
// operands are staged in their natural NHWC layout ([node][channel]) by a
// three-stage cp.async pipeline and transposed into the mma fragments by
// ldmatrix.trans.  Blocks of the first column tile also sum dY over their
// nodes (the bias gradient).
template <int BM>
__global__ void __launch_bounds__(kThreads) k_wgrad(WgradArgs a) {
  constexpr int WM = BM / 16, WN = 4 / WM, NT = 64 / WN / 8;
  constexpr int DS = BM + 8, XS = 64 + 8;   // row strides (bf16): conflict-free ldmatrix
  __shared__ __align__(16) bf16 Ds[kStages][kBK][DS];   // dY [node][co]
  __shared__ __align__(16) bf16 Xs[kStages][kBK][XS];   // X  [node][k]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp % WM, wn = warp / WM;
  const int K = 9 * a.cin;
  const int kb = blockIdx.x * 64, cb = blockIdx.y * BM;
  const int pbeg = blockIdx.z * a.chunk;
  const int pend = min(a.total, pbeg + a.chunk);
  const int nsteps = (pend - pbeg + kBK - 1) / kBK;
  const int dyN2 = a.dy_n * a.dy_n;
  const bool bias_block = blockIdx.x == 0;
  auto load_stage = [&](int s, int it) {
    const int pb = pbeg + it * kBK;
    for (int idx = tid; idx < kBK * (BM / 8); idx += kThreads) {
      const int pi = idx / (BM / 8), v = idx - pi * (BM / 8);
      const int p = pb + pi;
      const bf16* src = a.dy;
      const bool ok = p < pend;
      if (ok) {
        const int img = p / dyN2, q = p - img * dyN2;
        src = a.dy + (size_t)img * a.dy_img + (size_t)q * a.dy_cs + cb + 8 * v;
      }
      cp_async16(&Ds[s][pi][8 * v], src, ok ? 16 : 0);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int idx = tid + i * kThreads;   // 32 nodes x 8 groups of the 64 columns
      const int pi = idx >> 3, gg = idx & 7;
      const int p = pb + pi, k = kb + 8 * gg;
      const bf16* src = a.in;
      bool ok = p < pend && k < K;
      if (ok) {
        const int img = p / dyN2, q = p - img * dyN2;
        const int qy = q / a.dy_n, qx = q - qy * a.dy_n;
        const int tap = k / a.cin, ci = k - tap * a.cin;
        int sy, sx;
        ok = conv_src(0, a.stride, a.in_n, qy, qx, tap / 3 - 1, tap % 3 - 1, sy, sx);
        if (ok) src = a.in + (size_t)img * a.in_img + ((size_t)sy * a.in_n + sx) * a.in_cs + ci;
      }
      cp_async16(&Xs[s][pi][8 * gg], src, ok ? 16 : 0);
    }
  };
  float acc[NT][4];
#pragma unroll
  for (int j = 0; j < NT; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[j][e] = 0.f;
  float bsum = 0.f;
#pragma unroll
  for (int s = 0; s < kStages - 1; ++s) {
    if (s < nsteps) load_stage(s, s);
    cp_async_commit();
  }
  // ldmatrix.trans lane addresses: A (co x node) from Ds rows node, columns co;
  // B (node x k) from Xs rows node, columns k
  const int a_node = (lane & 7) + 8 * (lane >> 4), a_co = wm * 16 + 8 * ((lane >> 3) & 1);
  const int b_node = (lane & 7) + 8 * ((lane >> 3) & 1), b_k = wn * (64 / WN) + 8 * (lane >> 4);
  for (int it = 0; it < nsteps; ++it) {
    cp_async_wait<kStages - 2>();
    __syncthreads();
    {
      const int kn = it + kStages - 1;
      if (kn < nsteps) load_stage(kn % kStages, kn);
      cp_async_commit();
    }
    const int s = it % kStages;
    if (bias_block && tid < BM)
      for (int r = 0; r < kBK; ++r) bsum += __bfloat162float(Ds[s][r][tid]);
#pragma unroll
    for (int kk = 0; kk < kBK; kk += 16) {
      uint32_t af[4];
      ldsm_x4_trans(af, &Ds[s][kk + a_node][a_co]);
#pragma unroll
      for (int j = 0; j < NT; j += 2) {
        uint32_t bf[4];
        ldsm_x4_trans(bf, &Xs[s][kk + b_node][b_k + j * 8]);
        mma_bf16(acc[j], af, bf[0], bf[1]);
        mma_bf16(acc[j + 1], af, bf[2], bf[3]);
      }
    }
  }
  cp_async_wait<0>();
  float* part = a.part + (size_t)blockIdx.z * a.cout_pad * K;
#pragma unroll
  for (int j = 0; j < NT; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int co = cb + wm * 16 + (lane >> 2) + 8 * (e >> 1);
      const int k = kb + wn * (64 / WN) + j * 8 + 2 * (lane & 3) + (e & 1);
      if (k < K) part[(size_t)co * K + k] = acc[j][e];
    }
  if (bias_block && tid < BM) a.bpart[(size_t)blockIdx.z * a.cout_pad + cb + tid] = bsum;
}

// dW of one layer from the chunk partials, added in chunk order, into the
// flat gradient (W[cout][3][3][cin_real]); padding channels are dropped.
__global__ void k_wgrad_reduce(const float* part, int chunks, int cout, int cout_pad, int cin_real, int cin_pad,
                               float* grad) {
  const int n = cout * 9 * cin_real;
  const int K = 9 * cin_pad;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int co = i / (9 * cin_real), r = i - co * 9 * cin_real;
    const int tap = r / cin_real, ci = r - tap * cin_real;
    const size_t o = (size_t)co * K + tap * cin_pad + ci;
    float s = 0.f;
    for (int c = 0; c < chunks; ++c) s += part[(size_t)c * cout_pad * K + o];
    grad[i] = s;
  }
}

// the bias gradient from the chunks' node sums, in chunk order
__global__ void k_bgrad_reduce(const float* bpart, int chunks, int cout, int cout_pad, float* grad) {
  const int co = blockIdx.x * blockDim.x + threadIdx.x;
  if (co >= cout) return;
  float s = 0.f;
  for (int c = 0; c < chunks; ++c) s += bpart[(size_t)c * cout_pad + co];
  grad[co] = s;
}

// bilinear prolongation of node grids m -> 2m-1, C channels (C, channel
// strides and view offsets multiples of 8): one thread per node and group of
// 8 channels, 16-byte loads and stores
__global__ void k_up(const bf16* src, size_t src_img, int m, int src_cs, bf16* dst, size_t dst_img, int dst_cs,
                     int C, int images) {
  const int n = 2 * m - 1, G = C / 8;
  const size_t total = (size_t)images * n * n * G;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % G) * 8;
    const size_t node = i / G;
    const int img = (int)(node / ((size_t)n * n));
    const int q = (int)(node - (size_t)img * n * n);
    const int y = q / n, x = q - y * n;
    const bf16* s = src + (size_t)img * src_img + c;
    const int y0 = y >> 1, x0 = x >> 1, y1 = y0 + (y & 1), x1 = x0 + (x & 1);
    uint4 u[4];
    u[0] = *reinterpret_cast<const uint4*>(s + ((size_t)y0 * m + x0) * src_cs);
    u[1] = *reinterpret_cast<const uint4*>(s + ((size_t)y0 * m + x1) * src_cs);
    u[2] = *reinterpret_cast<const uint4*>(s + ((size_t)y1 * m + x0) * src_cs);
    u[3] = *reinterpret_cast<const uint4*>(s + ((size_t)y1 * m + x1) * src_cs);
    __align__(16) bf16 o[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      float v = __bfloat162float(reinterpret_cast<const bf16*>(&u[0])[e]);
      v += __bfloat162float(reinterpret_cast<const bf16*>(&u[1])[e]);
      v += __bfloat162float(reinterpret_cast<const bf16*>(&u[2])[e]);
      v += __bfloat162float(reinterpret_cast<const bf16*>(&u[3])[e]);
      o[e] = __float2bfloat16(0.25f * v);
    }
    *reinterpret_cast<uint4*>(dst + (size_t)img * dst_img + (size_t)q * dst_cs + c) =
        *reinterpret_cast<const uint4*>(o);
  }
}

// adjoint of k_up, times the ReLU mask of the coarse activation (8 channels per thread)
__global__ void k_up_back(const bf16* df, size_t df_img, int n, int df_cs, bf16* dc, size_t dc_img, int dc_cs,
                          const bf16* mask, size_t mask_img, int mask_cs, int C, int images) {
  const int m = (n + 1) / 2, G = C / 8;
  const size_t total = (size_t)images * m * m * G;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % G) * 8;
    const size_t node = i / G;
    const int img = (int)(node / ((size_t)m * m));
    const int q = (int)(node - (size_t)img * m * m);
    const int cy = q / m, cx = q - cy * m;
    const bf16* f = df + (size_t)img * df_img + c;
    float v[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) v[e] = 0.f;
#pragma unroll
    for (int a = -1; a <= 1; ++a)
#pragma unroll
      for (int b = -1; b <= 1; ++b) {
        const int y = 2 * cy + a, x = 2 * cx + b;
        if (y < 0 || y >= n || x < 0 || x >= n) continue;
        const float w = (a == 0 ? 1.f : 0.5f) * (b == 0 ? 1.f : 0.5f);
        const uint4 u = *reinterpret_cast<const uint4*>(f + ((size_t)y * n + x) * df_cs);
#pragma unroll
        for (int e = 0; e < 8; ++e) v[e] += w * __bfloat162float(reinterpret_cast<const bf16*>(&u)[e]);
      }
    const uint4 mu = *reinterpret_cast<const uint4*>(mask + (size_t)img * mask_img + (size_t)q * mask_cs + c);
    __align__(16) bf16 o[8];
#pragma unroll
    for (int e = 0; e < 8; ++e)
      o[e] = __float2bfloat16(__bfloat162float(reinterpret_cast<const bf16*>(&mu)[e]) > 0.f ? v[e] : 0.f);
    *reinterpret_cast<uint4*>(dc + (size_t)img * dc_img + (size_t)q * dc_cs + c) = *reinterpret_cast<const uint4*>(o);
  }
}

// network input: channels (R, T, 0 x 14) per node; R advances by r_stride per image (0 = shared)
__global__ void k_pack_input(const double* R, size_t r_stride, const double* T, size_t t_stride, int N, int images,
                             bf16* x) {
  const size_t total = (size_t)images * N;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t img = i / N, q = i - img * N;
    __align__(16) bf16 v[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) v[c] = __float2bfloat16(0.f);
    v[0] = __float2bfloat16((float)R[img * r_stride + q]);
    v[1] = __float2bfloat16((float)T[img * t_stride + q]);
    uint4* d = reinterpret_cast<uint4*>(x + i * 16);
    d[0] = reinterpret_cast<const uint4*>(v)[0];
    d[1] = reinterpret_cast<const uint4*>(v)[1];
  }
}

// loss = mean (out - target * scale)^2 over images, nodes, both channels;
// target [img][2][N] (component planes); gradient into dout (16 channels, 2 used).
// Per-block partial sums in a fixed order; k_loss_total adds them in block order.
__global__ void __launch_bounds__(256) k_mse(const float* out, const double* target, double scale, int N, int images,
                                             bf16* dout, float* part) {
  __shared__ float red[8];
  const size_t total = (size_t)images * N;
  const float inv = 1.f / (float)(2 * total);
  float s = 0.f;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t img = i / N, q = i - img * N;
    __align__(16) bf16 g[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) g[c] = __float2bfloat16(0.f);
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const float d = out[i * 2 + c] - (float)(target[(img * 2 + c) * N + q] * scale);
      s += d * d;
      g[c] = __float2bfloat16(2.f * d * inv);
    }
    uint4* dp = reinterpret_cast<uint4*>(dout + i * 16);
    dp[0] = reinterpret_cast<const uint4*>(g)[0];
    dp[1] = reinterpret_cast<const uint4*>(g)[1];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < 8; ++w) t += red[w];
    part[blockIdx.x] = t * inv;
  }
}
__global__ void k_loss_total(const float* part, int n, float* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    float s = 0.f;
    for (int i = 0; i < n; ++i) s += part[i];
    *out = s;
  }
}

// network output (pixels of its grid, node-major pairs) -> displacement planes in domain units
__global__ void k_out_to_phi(const float* out, double scale, int N, int images, double* phi) {
  const size_t total = (size_t)images * N;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t img = i / N, q = i - img * N;
    phi[(img * 2) * N + q] = (double)out[i * 2] * scale;
    phi[(img * 2 + 1) * N + q] = (double)out[i * 2 + 1] * scale;
  }
}

// Adam (Kingma & Ba 2015) on the fp32 master parameters
__global__ void k_adam(float* theta, const float* grad, float* m, float* v, int n, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float g = grad[i];
    const float mi = b1 * m[i] + (1.f - b1) * g;
    const float vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    theta[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// bf16 copies of one layer's weights: wf[cout_pad][tap][cin_pad] for the
// forward pass, wt[cin_pad][tap][cout_pad] for the data gradient
__global__ void k_pack_weights(const float* w, int cout, int cin, int cout_pad, int cin_pad, bf16* wf, bf16* wt) {
  const int n = cout_pad * 9 * cin_pad;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int co = i / (9 * cin_pad), r = i - co * 9 * cin_pad;
    const int tap = r / cin_pad, ci = r - tap * cin_pad;
    const float v = (co < cout && ci < cin) ? w[((size_t)co * 9 + tap) * cin + ci] : 0.f;
    const bf16 b = __float2bfloat16(v);
    wf[i] = b;
    wt[((size_t)ci * 9 + tap) * cout_pad + co] = b;
  }
}

}  // namespace unet
}  // namespace msg
