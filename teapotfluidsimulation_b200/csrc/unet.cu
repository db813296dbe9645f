// Learned preconditioner: a 3-level 3D convolutional U-Net (16/32/64 channels, 3^3 kernels, BF16
// weights and activations, FP32 accumulation), trained and applied with this file's own kernels.
//
// The network maps a residual field on a box of X x Y x Z cells (multiples of 4) to an approximate
// correction: input channels [r / s, liquid mask, air mask] with s = max |r| over the liquid cells,
// output z = s * net(...)[0] on the liquid cells (0 elsewhere). Layers (channels padded to multiples
// of 16; every conv 3^3, zero padding, bias, ReLU except the last):
//   enc1: 16->16, 16->16 (s1)        level 1 (X, Y, Z)
//   enc2: pool, 16->32, 32->32 (s2)  level 2 (X/2, ...), 2x2x2 average pooling
//   enc3: pool, 32->64, 64->64       level 3 (X/4, ...)
//   dec2: up, [up | s2] 96->32, 32->32     nearest-neighbour upsampling, channel concatenation
//   dec1: up, [up | s1] 48->16, 16->16
//   out : 16->16 (channel 0 used)
//
// Kernels (NDHWC activations, x fastest among the cells, channels innermost):
//  - k_conv_tc (default): implicit GEMM out[v][n] = bias[n] + sum_t sum_k in[v + off_t][k] G[t][n][k]
//    on the 5th-generation tensor cores (tcgen05.mma kind::f16, BF16 in, FP32 accumulator in tensor
//    memory), 128 cells x all output channels per CTA, operands staged per tap in shared memory by
//    asynchronous copies through L1 (the dx = -1, 0, +1 taps re-read nearly the same rows);
//    k_conv_tc_row, for boxes whose x extent is a multiple of 128, instead streams 16 rows per CTA
//    through a ring of input-row windows. k_conv computes the same on the warp-level path (mma.sync
//    m16n8k16, one warp per 16 cells), kept for comparison (pl_unet_set_conv_kernel). Both compute the
//    data gradient with G[t][n][k] = W[26 - t][n][k] (flipped taps).
//  - k_wgrad: weight gradient dW[t][ci][co] = sum_v in[v + off_t][ci] d[v][co] on the tensor cores:
//    a CTA stages a chunk of cells of both operands transposed in shared memory ([channel][cell]) and
//    accumulates the Cin x Cout tile; per-chunk partials are summed in a fixed order (deterministic).
//  - pooling, upsampling, concatenation, ReLU masks, the loss and Adam are elementwise kernels.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "unet.h"

namespace pl {

namespace {

typedef __nv_bfloat16 bf16;

constexpr int NLAYER = 11;
constexpr int WG_CHUNK = 2048;  // cells per weight-gradient CTA
constexpr int WG_KC = 32;       // cells per shared-memory stage of the weight gradient

struct LayerSpec {
  int cin, cout;
};
constexpr LayerSpec SPEC[NLAYER] = {{16, 16}, {16, 16}, {16, 32}, {32, 32}, {32, 64}, {64, 64},
                                    {96, 32}, {32, 32}, {48, 16}, {16, 16}, {16, 16}};

__device__ __forceinline__ uint32_t ld32(const bf16* p) { return *reinterpret_cast<const uint32_t*>(p); }

__device__ __forceinline__ void mma16816(float* c, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

struct Box {
  int X, Y, Z, count;
  __host__ __device__ int cells() const { return X * Y * Z; }
  __host__ __device__ int total() const { return X * Y * Z * count; }
};

// Cell index of the neighbour of cell v (global over the batch) at tap t (offsets -1..1, tap = dz*9 +
// dy*3 + dx), or -1 outside the box.
__device__ __forceinline__ int tap_cell(const Box& B, int v, int t) {
  const int per = B.cells();
  const int s = v / per;
  const int c = v - s * per;
  const int x = c % B.X, y = (c / B.X) % B.Y, z = c / (B.X * B.Y);
  const int xx = x + t % 3 - 1, yy = y + (t / 3) % 3 - 1, zz = z + t / 9 - 1;
  if (xx < 0 || yy < 0 || zz < 0 || xx >= B.X || yy >= B.Y || zz >= B.Z) return -1;
  return s * per + (zz * B.Y + yy) * B.X + xx;
}

// Implicit-GEMM 3^3 convolution on NDHWC BF16 tensors. One warp per 16 output cells, all NOUT output
// channels (NOUT = 16, 32 or 64: NOUT / 8 tiles of 8); K = 27 taps x CIN input channels in steps of 16.
// out_f32 (optional): FP32 result; out_bf (optional): BF16 result after the optional ReLU; mask
// (optional): the result is multiplied by (mask > 0) (the ReLU of the layer that produced the input
// whose gradient this is).
template <int NOUT>
__global__ void __launch_bounds__(128) k_conv(Box B, const bf16* __restrict__ in, int cin, const bf16* __restrict__ G,
                                              const float* __restrict__ bias, int relu, const bf16* __restrict__ mask,
                                              bf16* out_bf, float* out_f32) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31, g = lane >> 2, tg = lane & 3;
  const int v0 = warp * 16;
  const int total = B.total();
  if (v0 >= total) return;
  constexpr int NT = NOUT / 8;
  float acc[NT][4];
#pragma unroll
  for (int j = 0; j < NT; j++) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
  const int va = v0 + g, vb = v0 + g + 8;  // the two rows this lane feeds
  for (int t = 0; t < 27; t++) {
    const int na = va < total ? tap_cell(B, va, t) : -1;
    const int nb = vb < total ? tap_cell(B, vb, t) : -1;
    const bf16* pa = na >= 0 ? in + (size_t)na * cin : nullptr;
    const bf16* pb = nb >= 0 ? in + (size_t)nb * cin : nullptr;
    const bf16* gt = G + (size_t)t * NOUT * cin;
    for (int k0 = 0; k0 < cin; k0 += 16) {
      const uint32_t a0 = pa ? ld32(pa + k0 + 2 * tg) : 0u;
      const uint32_t a1 = pb ? ld32(pb + k0 + 2 * tg) : 0u;
      const uint32_t a2 = pa ? ld32(pa + k0 + 2 * tg + 8) : 0u;
      const uint32_t a3 = pb ? ld32(pb + k0 + 2 * tg + 8) : 0u;
#pragma unroll
      for (int j = 0; j < NT; j++) {
        const bf16* gb = gt + (size_t)(j * 8 + g) * cin + k0 + 2 * tg;
        mma16816(acc[j], a0, a1, a2, a3, ld32(gb), ld32(gb + 8));
      }
    }
  }
#pragma unroll
  for (int j = 0; j < NT; j++) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int v = h ? vb : va;
      if (v >= total) continue;
      const int n = j * 8 + 2 * tg;
      float r0 = acc[j][2 * h], r1 = acc[j][2 * h + 1];
      if (bias) {
        r0 += bias[n];
        r1 += bias[n + 1];
      }
      if (relu) {
        r0 = fmaxf(r0, 0.f);
        r1 = fmaxf(r1, 0.f);
      }
      if (mask) {
        const bf16* m = mask + (size_t)v * NOUT + n;
        if (!(__bfloat162float(m[0]) > 0.f)) r0 = 0.f;
        if (!(__bfloat162float(m[1]) > 0.f)) r1 = 0.f;
      }
      if (out_f32) {
        out_f32[(size_t)v * NOUT + n] = r0;
        out_f32[(size_t)v * NOUT + n + 1] = r1;
      }
      if (out_bf) {
        __nv_bfloat162 p;
        p.x = __float2bfloat16(r0);
        p.y = __float2bfloat16(r1);
        *reinterpret_cast<__nv_bfloat162*>(out_bf + (size_t)v * NOUT + n) = p;
      }
    }
  }
}

// ---------------------------------------------------------------- tcgen05 convolution (sm_100a)
//
// The same implicit GEMM on the 5th-generation tensor cores: one CTA of 128 threads per 128 output
// cells (M = 128), all NOUT output channels (N), K = 27 taps x CIN in MMAs of K = 16. Per tap the CTA
// stages the 128 gathered input rows (A: cells x CIN) and the tap's weights (B: NOUT x CIN) in shared
// memory in the canonical K-major layout without swizzle (8-row x 16-byte core matrices; cores
// adjacent in K 128 bytes apart, cores adjacent in M/N 256 bytes apart), then one thread issues the
// tap's MMAs into an FP32 accumulator in tensor memory and commits them to the buffer's mbarrier.
// Two buffers: the staging of tap t + 1 overlaps the MMAs of tap t. The epilogue reads the
// accumulator back with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = rows of its cells).
// Every mbarrier wait is bounded: on a timeout the CTA sets *err, stops issuing, waits (bounded) for
// its MMAs in flight, frees its tensor memory and returns.

constexpr int TC_SPIN = 1 << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (sm_100 format): start address, leading (K) and stride (M/N) byte
// offsets, all in 16-byte units; descriptor version 1; no swizzle.
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr & 0x3FFFF) >> 4) | ((uint64_t)((lbo & 0x3FFFF) >> 4) << 16) |
         ((uint64_t)((sbo & 0x3FFFF) >> 4) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major, N, M = 128.
template <int N>
__host__ __device__ constexpr uint32_t tc_idesc() {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ bool tc_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (int i = 0; i < TC_SPIN; i++) {
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

// Independent accumulators per output tile: tap t accumulates into accumulator t mod TC_NACC, so that
// consecutive MMAs do not wait on each other's result (a chain of small MMAs into one accumulator is
// bound by the MMA latency, not its throughput); the epilogue sums them in a fixed order.
template <int NOUT>
__host__ __device__ constexpr int tc_nacc() {
  return NOUT <= 32 ? 4 : NOUT <= 64 ? 2 : 1;
}

// Host copies of tc_cols / tc_nacc for run-time channel counts (shared-memory sizing).
inline int tc_ncol(int cols) { return cols <= 32 ? 32 : cols <= 64 ? 64 : cols <= 128 ? 128 : cols <= 256 ? 256 : 512; }
inline int tc_nacc_h(int nout) { return nout <= 32 ? 4 : nout <= 64 ? 2 : 1; }

template <int NOUT>
__host__ __device__ constexpr int tc_cols() {  // power of two >= 32 that holds NOUT columns
  return NOUT <= 32 ? 32 : NOUT <= 64 ? 64 : NOUT <= 128 ? 128 : NOUT <= 256 ? 256 : 512;
}

// Sum of NACC accumulators (NOUT columns apart) for 16 columns of this warp's 32 lanes, in
// accumulator order.
template <int NACC, int NOUT>
__device__ __forceinline__ void tc_ld_sum(uint32_t taddr, float* sum) {
#pragma unroll
  for (int a = 0; a < NACC; a++) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr + (uint32_t)(a * NOUT)));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 16; q++) sum[q] = a ? sum[q] + __uint_as_float(r[q]) : __uint_as_float(r[q]);
  }
}

constexpr int TC_STAGES = 4;  // (A, B) stages in flight: taps t + 1 .. t + 3 load while tap t multiplies

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}

template <int NOUT>
__global__ void __launch_bounds__(128) k_conv_tc(Box B, const bf16* __restrict__ in, int cin,
                                                 const bf16* __restrict__ G, const float* __restrict__ bias, int relu,
                                                 const bf16* __restrict__ mask, bf16* out_bf, float* out_f32,
                                                 int* err) {
  extern __shared__ __align__(1024) uint8_t smem[];
  constexpr int NACC = 1;  // one accumulator and one issuing thread: more resident CTAs
  constexpr int NCOL = tc_cols<NACC * NOUT>();
  constexpr uint32_t IDESC = tc_idesc<NOUT>();
  constexpr int S = TC_STAGES;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int total = B.total();
  const int v0 = blockIdx.x * 128;
  const int a_bytes = 128 * cin * 2, b_bytes = NOUT * cin * 2;
  const int stage_bytes = a_bytes + b_bytes;
  const uint32_t sbase = smem_u32(smem);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + S * stage_bytes);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + S);
  if (tid == 0) {
    for (int q = 0; q < S; q++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[q])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(NCOL)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  const int v = v0 + tid;
  const int kch = cin / 8;  // 16-byte chunks per row
  // this thread's cell, decomposed once (the taps only add offsets and test the box faces)
  const int per = B.cells(), XY = B.X * B.Y;
  const int cl = v < total ? v % per : 0;
  const int cx = cl % B.X, cy = (cl / B.X) % B.Y, cz = cl / XY;
  // this thread's share of a tap's weights, at most TC_BMAX 16-byte chunks: shared- and global-memory
  // offsets computed once
  constexpr int TC_BMAX = (NOUT * 12 + 127) / 128;  // Cin <= 96
  uint32_t boff[TC_BMAX];
  int goff[TC_BMAX];
  const int nbch = NOUT * kch;
#pragma unroll
  for (int q = 0; q < TC_BMAX; q++) {
    const int e = tid + 128 * q;
    const int n = e / kch, c = e - n * kch;
    boff[q] = (c >> 1) * (NOUT * 32) + ((n >> 3) * 2 + (c & 1)) * 128 + (n & 7) * 16;
    goff[q] = n * cin + 8 * c;
  }
  // stage s <- tap t: this thread's gathered row (zero-filled outside the box) and its share of the
  // tap's weights, as 16-byte asynchronous copies, one commit group per tap
  auto load_tap = [&](int t, int s) {
    const uint32_t a0 = sbase + s * stage_bytes, b0 = a0 + a_bytes;
    const int dx = t % 3 - 1, dy = (t / 3) % 3 - 1, dz = t / 9 - 1;
    const bool in_box = v < total && (unsigned)(cx + dx) < (unsigned)B.X && (unsigned)(cy + dy) < (unsigned)B.Y &&
                        (unsigned)(cz + dz) < (unsigned)B.Z;
    const bf16* src = in_box ? in + (size_t)(v + dx + dy * B.X + dz * XY) * cin : in;
    const uint32_t nbytes = in_box ? 16u : 0u;
    const uint32_t arow = a0 + (tid >> 3) * 256 + (tid & 7) * 16;
    for (int c = 0; c < kch; c++) cp_async16(arow + (c >> 1) * 4096 + (c & 1) * 128, src + 8 * c, nbytes);
    const bf16* gt = G + (size_t)t * NOUT * cin;
#pragma unroll
    for (int q = 0; q < TC_BMAX; q++)
      if (tid + 128 * q < nbch) cp_async16(b0 + boff[q], gt + goff[q], 16u);
  };
  for (int p = 0; p < S - 1; p++) {
    load_tap(p, p);
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  bool bad = false;
  bool timed_out = false;
  int issued = 0;  // taps whose MMAs were issued
  for (int t = 0; t < 27; t++) {
    const int s = t % S;
    asm volatile("cp.async.wait_group %0;" ::"n"(S - 2) : "memory");  // this thread's copies of tap t landed
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");      // ... and are visible to the MMA
    if (__syncthreads_or(bad ? 1 : 0)) {
      timed_out = true;
      break;
    }
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = sbase + s * stage_bytes, b0 = a0 + a_bytes;
      for (int kc = 0; kc < cin / 16; kc++) {
        const uint64_t ad = tc_desc(a0 + kc * 4096, 128, 256);
        const uint64_t bd = tc_desc(b0 + kc * (NOUT * 32), 128, 256);
        const uint32_t acc = (t | kc) != 0 ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(IDESC), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&mbar[s]))
                   : "memory");
    }
    issued = t + 1;
    const int tn = t + S - 1;
    if (tn < 27) {
      const int sn = tn % S;  // = (t - 1) % S: free once the MMAs of tap t - 1 are done
      if (t >= 1) bad = !tc_wait(&mbar[sn], uint32_t(((t - 1) / S) & 1));
      if (!bad) load_tap(tn, sn);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");  // (empty past the last tap: keeps the count)
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  // the last commit tracks every MMA issued before it
  bool done = true;
  if (issued > 0) {
    const int tl = issued - 1;
    done = tc_wait(&mbar[tl % S], uint32_t((tl / S) & 1));
  }
  if (__syncthreads_or(done ? 0 : 1)) timed_out = true;
  if (timed_out) {
    if (tid == 0) atomicExch(err, 1);
  } else {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
    for (int c0 = 0; c0 < NOUT; c0 += 16) {
      float sum[16];
      tc_ld_sum<NACC, NOUT>(lane_base + (uint32_t)c0, sum);
      const int vr = v0 + warp * 32 + lane;
      if (vr < total) {
        float f[16];
#pragma unroll
        for (int q = 0; q < 16; q++) {
          float x = sum[q];
          if (bias) x += bias[c0 + q];
          if (relu) x = fmaxf(x, 0.f);
          if (mask && !(__bfloat162float(mask[(size_t)vr * NOUT + c0 + q]) > 0.f)) x = 0.f;
          f[q] = x;
        }
        if (out_f32) {
          float4* o = reinterpret_cast<float4*>(out_f32 + (size_t)vr * NOUT + c0);
#pragma unroll
          for (int q = 0; q < 4; q++) o[q] = make_float4(f[4 * q], f[4 * q + 1], f[4 * q + 2], f[4 * q + 3]);
        }
        if (out_bf) {
          __align__(16) bf16 h[16];
#pragma unroll
          for (int q = 0; q < 16; q++) h[q] = __float2bfloat16(f[q]);
          uint4* o = reinterpret_cast<uint4*>(out_bf + (size_t)vr * NOUT + c0);
          o[0] = *reinterpret_cast<uint4*>(&h[0]);
          o[1] = *reinterpret_cast<uint4*>(&h[8]);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCOL) : "memory");
  }
}

// Row-tile variant for boxes whose x extent is a multiple of 128. A CTA owns a 128-cell segment
// (x0..x0+127) of TC_RROWS consecutive rows y0..y0+R-1 at fixed z of one box and walks along y: for
// output row y it needs the input rows y-1, y, y+1 at z-1, z, z+1, each as a window of 130 cells
// (x0-1..x0+128, zero outside the box). Windows live in a 4-slot ring indexed by y mod 4 (3 windows,
// one per dz, per slot), so while the MMAs of row y read slots y-1..y+1 the copies of row y+2 fill
// the fourth: every input row is staged once per CTA instead of 27 times. Tap (dx, dy, dz) is the
// window (y+dy, dz) read from row dx: a shared-memory descriptor shifted by dx rows (a window holds,
// per 8-channel group, 130 rows of 16 bytes back to back: 8-row groups 128 B apart, the next group
// 2080 B on). All 27 taps' weights are staged once per CTA. The taps go round-robin into NACC
// independent accumulators, each issued by its own warp (one tcgen05.mma issue costs a few hundred
// cycles, so a single issuing thread was the row's critical path); the accumulators of a row are read
// back (tcgen05.ld) while the next row's MMAs fill a second set.
constexpr int TC_WROWS = 130;
constexpr int TC_RROWS = 16;

template <int CIN, int NOUT>
__global__ void __launch_bounds__(128) k_conv_tc_row(Box B, const bf16* __restrict__ in, int,
                                                     const bf16* __restrict__ G, const float* __restrict__ bias,
                                                     int relu, const bf16* __restrict__ mask, bf16* out_bf,
                                                     float* out_f32, int* err) {
  extern __shared__ __align__(1024) uint8_t smem[];
  constexpr int NACC = tc_nacc<NOUT>();
  constexpr int NCOL = tc_cols<2 * NACC * NOUT>();  // two rows' accumulator sets
  constexpr uint32_t IDESC = tc_idesc<NOUT>();
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr int cin = CIN, kch = CIN / 8;
  const int win_bytes = kch * TC_WROWS * 16;  // one window (one input row, one dz)
  const int slot_bytes = 3 * win_bytes;       // the three dz windows of one input row y
  constexpr int tap_bytes = NOUT * CIN * 2;  // one tap's weights
  const uint32_t sbase = smem_u32(smem);
  const uint32_t bbase = sbase + 4 * slot_bytes;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + 4 * slot_bytes + 27 * tap_bytes);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 2);
  // CTA -> (box, z, row block, x segment)
  const int xseg = B.X / 128, yblk = (B.Y + TC_RROWS - 1) / TC_RROWS;
  int b = blockIdx.x;
  const int xs = b % xseg;
  b /= xseg;
  const int yb = b % yblk;
  b /= yblk;
  const int z = b % B.Z, sb = b / B.Z;
  const int x0 = xs * 128, y0 = yb * TC_RROWS, y1 = min(B.Y, y0 + TC_RROWS);
  const size_t box0 = (size_t)sb * B.cells();
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar[0])), "r"(NACC) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar[1])), "r"(NACC) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(NCOL)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  }
  // input row yy (all three dz) into its ring slot; chunk e = (dz, row, c), c fastest, so consecutive
  // threads read consecutive 16-byte chunks (a cell's channels, then the next cell's)
  const int wchunks = TC_WROWS * kch;
  auto load_row = [&](int yy) {
    const uint32_t slot = sbase + (yy & 3) * slot_bytes;
    for (int e = tid; e < 3 * wchunks; e += 128) {
      const int w = e / wchunks, rem = e - w * wchunks;
      const int row = rem / kch, c = rem - row * kch;
      const int zz = z + w - 1, xx = x0 - 1 + row;
      const bool ok = (unsigned)yy < (unsigned)B.Y && (unsigned)zz < (unsigned)B.Z && (unsigned)xx < (unsigned)B.X;
      const bf16* src = ok ? in + (box0 + (size_t)(zz * B.Y + yy) * B.X + xx) * cin + 8 * c : in;
      cp_async16(slot + w * win_bytes + c * (TC_WROWS * 16) + row * 16, src, ok ? 16u : 0u);
    }
  };
  for (int e = tid; e < 27 * NOUT * kch; e += 128) {  // all 27 taps' weights, canonical layout
    const int t = e / (NOUT * kch), rem = e - t * (NOUT * kch);
    const int n = rem / kch, c = rem - n * kch;
    cp_async16(bbase + t * tap_bytes + (c >> 1) * (NOUT * 32) + ((n >> 3) * 2 + (c & 1)) * 128 + (n & 7) * 16,
               G + (size_t)t * NOUT * cin + (size_t)n * cin + 8 * c, 16u);
  }
  load_row(y0 - 1);
  load_row(y0);
  load_row(y0 + 1);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  // two sets of NACC accumulators (row parity): the MMAs of row y run while the epilogue of row y - 1
  // reads the other set
  auto epilogue = [&](int y, uint32_t acc_col) {
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16) + acc_col;
    const size_t vr = box0 + (size_t)(z * B.Y + y) * B.X + x0 + warp * 32 + lane;
#pragma unroll
    for (int c0 = 0; c0 < NOUT; c0 += 16) {
      float sum[16];
      tc_ld_sum<NACC, NOUT>(lane_base + (uint32_t)c0, sum);
      float f[16];
#pragma unroll
      for (int q = 0; q < 16; q++) {
        float x = sum[q];
        if (bias) x += bias[c0 + q];
        if (relu) x = fmaxf(x, 0.f);
        if (mask && !(__bfloat162float(mask[vr * NOUT + c0 + q]) > 0.f)) x = 0.f;
        f[q] = x;
      }
      if (out_f32) {
        float4* o = reinterpret_cast<float4*>(out_f32 + vr * NOUT + c0);
#pragma unroll
        for (int q = 0; q < 4; q++) o[q] = make_float4(f[4 * q], f[4 * q + 1], f[4 * q + 2], f[4 * q + 3]);
      }
      if (out_bf) {
        __align__(16) bf16 h[16];
#pragma unroll
        for (int q = 0; q < 16; q++) h[q] = __float2bfloat16(f[q]);
        uint4* o = reinterpret_cast<uint4*>(out_bf + vr * NOUT + c0);
        o[0] = *reinterpret_cast<uint4*>(&h[0]);
        o[1] = *reinterpret_cast<uint4*>(&h[8]);
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");  // reads done before that buffer's next MMAs
  };
  bool failed = false;
  int last = -1;  // row whose accumulator still waits for its epilogue
  for (int y = y0; y < y1; y++) {
    const int k = y - y0;
    asm volatile("cp.async.wait_all;" ::: "memory");  // rows y-1..y+1 (and the weights) landed
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();  // also: the epilogue of row y - 2 (the same accumulator) has read it
    if (lane == 0 && warp < NACC) {  // warp a issues the taps of accumulator a (t = a mod NACC)
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t dacc = tmem + (uint32_t)((k & 1) * NACC * NOUT + warp * NOUT);
      for (int t = warp; t < 27; t += NACC) {
        const int dy = (t / 3) % 3, dz = t / 9, dx = t % 3;  // each 0..2 (offset + 1)
        const uint32_t wa = sbase + ((y - 1 + dy) & 3) * slot_bytes + dz * win_bytes + dx * 16;
#pragma unroll
        for (int kc = 0; kc < CIN / 16; kc++) {
          const uint64_t ad = tc_desc(wa + (2 * kc) * (TC_WROWS * 16), TC_WROWS * 16, 128);
          const uint64_t bd = tc_desc(bbase + t * tap_bytes + kc * (NOUT * 32), 128, 256);
          const uint32_t acc = (t >= NACC || kc != 0) ? 1u : 0u;
          asm volatile(
              "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
              " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(dacc),
              "l"(ad), "l"(bd), "r"(IDESC), "r"(acc)
              : "memory");
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&mbar[k & 1]))
                   : "memory");
    }
    if (last >= 0) {
      // row y - 1: its MMAs done, then its ring slot (y - 2) & 3 is free for row y + 2 and its
      // accumulator can be read
      const int kl = last - y0;
      const bool done = tc_wait(&mbar[kl & 1], uint32_t((kl >> 1) & 1));
      if (__syncthreads_or(done ? 0 : 1)) {
        failed = true;
        break;
      }
      if (y + 1 < y1) load_row(y + 2);
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      epilogue(last, (uint32_t)((kl & 1) * NACC * NOUT));
    } else if (y + 1 < y1) {
      load_row(y + 2);  // slot (y0 + 2) & 3 has not been used
    }
    last = y;
  }
  if (!failed && last >= 0) {
    const int kl = last - y0;
    const bool done = tc_wait(&mbar[kl & 1], uint32_t((kl >> 1) & 1));
    if (__syncthreads_or(done ? 0 : 1)) {
      failed = true;
    } else {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      epilogue(last, (uint32_t)((kl & 1) * NACC * NOUT));
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  if (failed) {
    if (tid == 0) atomicExch(err, 1);
    for (int q = 0; q < 2; q++) tc_wait(&mbar[q], 0u), tc_wait(&mbar[q], 1u);  // MMAs in flight (bounded)
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCOL) : "memory");
  }
}

// Shared memory of k_conv_tc_row: the 4 ring slots (3 windows each), 27 taps' weights, the mbarrier
// and the TMEM address; with the floor of k_conv_tc so that the resident CTAs fit the SM's
// tensor-memory columns.
inline size_t tc_row_smem(int cin, int nout) {
  const size_t need = size_t(12) * (cin / 8) * TC_WROWS * 16 + size_t(27) * nout * cin * 2 + 64;
  const int ncol = tc_ncol(2 * tc_nacc_h(nout) * nout);  // two rows' accumulator sets
  const size_t floor_b = size_t(233472) / size_t(512 / ncol) + 1024;
  return std::max(need, ncol > 32 ? floor_b : need);
}

inline unsigned tc_row_blocks(const Box& B) {
  return unsigned((B.X / 128) * ((B.Y + TC_RROWS - 1) / TC_RROWS) * B.Z * B.count);
}

// Dynamic shared memory of k_conv_tc: TC_STAGES (A, B) stages, the mbarriers and the TMEM address; at
// least enough that no more CTAs share an SM than its 512 tensor-memory columns serve.
inline size_t tc_smem(int cin, int nout) {
  const size_t need = TC_STAGES * (size_t(128) * cin * 2 + size_t(nout) * cin * 2) + 8 * TC_STAGES + 64;
  const int ncol = tc_ncol(nout);
  const size_t floor_b = size_t(233472) / size_t(512 / ncol) + 1024;
  return std::max(need, ncol > 32 ? floor_b : need);
}

// Weight gradient of one tap t = blockIdx.y: part[chunk][t][ci][co] = sum over the CTA's cells v of
// in[v + off_t][ci] d[v][co]. Shared memory holds WG_KC cells of both operands transposed
// ([channel][cell]), so the A fragment (row = ci, k = cell) and the B fragment (k = cell, col = co) read
// consecutive cells. 4 warps; warp w owns the 16-row blocks w, w + 4 of Cin (CIN <= 96: 6 blocks).
template <int CIN, int COUT>
__global__ void __launch_bounds__(128) k_wgrad(Box B, const bf16* __restrict__ in, const bf16* __restrict__ d,
                                               float* part) {
  constexpr int MB = CIN / 16, NT = COUT / 8;
  constexpr int LD = WG_KC + 8;  // padded row (cells) in shared memory
  __shared__ __align__(16) bf16 sa[CIN * LD];
  __shared__ __align__(16) bf16 sb[COUT * LD];
  const int t = blockIdx.y;
  const int total = B.total();
  const int c0 = blockIdx.x * WG_CHUNK;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tg = lane & 3;
  float acc[2][NT][4];
#pragma unroll
  for (int m = 0; m < 2; m++)
#pragma unroll
    for (int j = 0; j < NT; j++) acc[m][j][0] = acc[m][j][1] = acc[m][j][2] = acc[m][j][3] = 0.f;
  for (int base = c0; base < min(c0 + WG_CHUNK, total); base += WG_KC) {
    __syncthreads();
    // stage: thread -> (cell, channel pair)
    for (int e = threadIdx.x; e < WG_KC * (CIN / 2); e += blockDim.x) {
      const int k = e / (CIN / 2), cp = (e % (CIN / 2)) * 2;
      const int v = base + k;
      const int nv = v < total ? tap_cell(B, v, t) : -1;
      bf16 x0 = __float2bfloat16(0.f), x1 = x0;
      if (nv >= 0) {
        x0 = in[(size_t)nv * CIN + cp];
        x1 = in[(size_t)nv * CIN + cp + 1];
      }
      sa[cp * LD + k] = x0;
      sa[(cp + 1) * LD + k] = x1;
    }
    for (int e = threadIdx.x; e < WG_KC * (COUT / 2); e += blockDim.x) {
      const int k = e / (COUT / 2), cp = (e % (COUT / 2)) * 2;
      const int v = base + k;
      bf16 y0 = __float2bfloat16(0.f), y1 = y0;
      if (v < total) {
        y0 = d[(size_t)v * COUT + cp];
        y1 = d[(size_t)v * COUT + cp + 1];
      }
      sb[cp * LD + k] = y0;
      sb[(cp + 1) * LD + k] = y1;
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < WG_KC; ks += 16) {
#pragma unroll
      for (int m = 0; m < 2; m++) {
        const int mb = warp + 4 * m;
        if (mb >= MB) continue;
        const bf16* ra = sa + (mb * 16 + g) * LD + ks + 2 * tg;
        const bf16* rb = sa + (mb * 16 + g + 8) * LD + ks + 2 * tg;
        const uint32_t a0 = ld32(ra), a1 = ld32(rb), a2 = ld32(ra + 8), a3 = ld32(rb + 8);
#pragma unroll
        for (int j = 0; j < NT; j++) {
          const bf16* cb = sb + (j * 8 + g) * LD + ks + 2 * tg;
          mma16816(acc[m][j], a0, a1, a2, a3, ld32(cb), ld32(cb + 8));
        }
      }
    }
  }
  float* out = part + ((size_t)blockIdx.x * 27 + t) * CIN * COUT;
#pragma unroll
  for (int m = 0; m < 2; m++) {
    const int mb = warp + 4 * m;
    if (mb >= MB) continue;
#pragma unroll
    for (int j = 0; j < NT; j++) {
      const int ci = mb * 16 + g, co = j * 8 + 2 * tg;
      out[ci * COUT + co] = acc[m][j][0];
      out[ci * COUT + co + 1] = acc[m][j][1];
      out[(ci + 8) * COUT + co] = acc[m][j][2];
      out[(ci + 8) * COUT + co + 1] = acc[m][j][3];
    }
  }
}

// dW[i] = sum over chunks (fixed order) of part[chunk][i]; db[co] = sum of the per-chunk bias sums.
__global__ void k_wgrad_reduce(const float* part, int nchunk, int n, float* dw) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = 0.f;
  for (int c = 0; c < nchunk; c++) s += part[(size_t)c * n + i];
  dw[i] = s;
}

// Bias gradient: db[co] = sum over cells of d[v][co], per-block partials (fixed order) then summed.
__global__ void k_bgrad_part(Box B, const bf16* d, int cout, float* part) {
  const int co = threadIdx.x % cout, lanes = blockDim.x / cout, sub = threadIdx.x / cout;
  const int total = B.total();
  const int c0 = blockIdx.x * WG_CHUNK;
  float s = 0.f;
  for (int v = c0 + sub; v < min(c0 + WG_CHUNK, total); v += lanes) s += __bfloat162float(d[(size_t)v * cout + co]);
  __shared__ float sh[256];
  sh[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x < cout) {
    float a = 0.f;
    for (int q = 0; q < lanes; q++) a += sh[q * cout + threadIdx.x];
    part[(size_t)blockIdx.x * cout + threadIdx.x] = a;
  }
}

// 2x2x2 average pooling (fine box F -> coarse box C = F / 2).
__global__ void k_pool(Box F, Box Cb, const bf16* in, int c, bf16* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Cb.total() * c) return;
  const int ch = i % c, v = i / c;
  const int per = Cb.cells(), s = v / per, cc = v % per;
  const int x = cc % Cb.X, y = (cc / Cb.X) % Cb.Y, z = cc / (Cb.X * Cb.Y);
  float a = 0.f;
#pragma unroll
  for (int q = 0; q < 8; q++) {
    const int fv = s * F.cells() + ((2 * z + (q >> 2)) * F.Y + 2 * y + ((q >> 1) & 1)) * F.X + 2 * x + (q & 1);
    a += __bfloat162float(in[(size_t)fv * c + ch]);
  }
  out[(size_t)v * c + ch] = __float2bfloat16(a * 0.125f);
}

// Gradient of the pooling: every fine cell gets 1/8 of its parent's gradient, added to dst (fine).
__global__ void k_pool_bwd_add(Box F, Box Cb, const bf16* dc, int c, bf16* dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= F.total() * c) return;
  const int ch = i % c, v = i / c;
  const int per = F.cells(), s = v / per, cc = v % per;
  const int x = cc % F.X, y = (cc / F.X) % F.Y, z = cc / (F.X * F.Y);
  const int pv = s * Cb.cells() + ((z >> 1) * Cb.Y + (y >> 1)) * Cb.X + (x >> 1);
  const float g = __bfloat162float(dc[(size_t)pv * c + ch]) * 0.125f;
  dst[i] = __float2bfloat16(__bfloat162float(dst[i]) + g);
}

// Nearest-neighbour upsampling of a (coarse, cu channels) into channels [0, cu) of a concatenation of
// width ctot, and the skip tensor (fine, cs channels) into channels [cu, ctot).
__global__ void k_up_concat(Box F, Box Cb, const bf16* coarse, int cu, const bf16* skip, int cs, bf16* out) {
  const int ctot = cu + cs, q8 = ctot / 8;  // 16-byte chunks per output cell (channels are multiples of 16)
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)F.total() * q8) return;
  const int q = int(i % q8), v = int(i / q8);
  const int ch = q * 8;
  uint4 val;
  if (ch >= cu) {
    val = *reinterpret_cast<const uint4*>(skip + (size_t)v * cs + ch - cu);
  } else {
    const int per = F.cells(), s = v / per, cc = v % per;
    const int x = cc % F.X, y = (cc / F.X) % F.Y, z = cc / (F.X * F.Y);
    const int pv = s * Cb.cells() + ((z >> 1) * Cb.Y + (y >> 1)) * Cb.X + (x >> 1);
    val = *reinterpret_cast<const uint4*>(coarse + (size_t)pv * cu + ch);
  }
  *reinterpret_cast<uint4*>(out + (size_t)v * ctot + ch) = val;
}

// Gradient of k_up_concat: the coarse part sums its 8 children (masked by the coarse activation's
// ReLU), the skip part is added to dskip.
__global__ void k_up_concat_bwd_coarse(Box F, Box Cb, const bf16* dcat, int cu, int ctot, const bf16* act,
                                       bf16* dcoarse) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Cb.total() * cu) return;
  const int ch = i % cu, v = i / cu;
  const int per = Cb.cells(), s = v / per, cc = v % per;
  const int x = cc % Cb.X, y = (cc / Cb.X) % Cb.Y, z = cc / (Cb.X * Cb.Y);
  float a = 0.f;
#pragma unroll
  for (int q = 0; q < 8; q++) {
    const int fv = s * F.cells() + ((2 * z + (q >> 2)) * F.Y + 2 * y + ((q >> 1) & 1)) * F.X + 2 * x + (q & 1);
    a += __bfloat162float(dcat[(size_t)fv * ctot + ch]);
  }
  if (!(__bfloat162float(act[i]) > 0.f)) a = 0.f;
  dcoarse[i] = __float2bfloat16(a);
}

__global__ void k_concat_bwd_skip(int total, const bf16* dcat, int cu, int ctot, int cs, bf16* dskip) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total * cs) return;
  const int ch = i % cs, v = i / cs;
  dskip[i] = dcat[(size_t)v * ctot + cu + ch];
}

// d = d * (act > 0)
__global__ void k_relu_mask(int n, bf16* d, const bf16* act) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (!(__bfloat162float(act[i]) > 0.f)) d[i] = __float2bfloat16(0.f);
}

// Per-sample scale s = max |r| over the liquid cells and, with e, the target energy sum e^2, in two
// passes with a fixed order: STAT_BLOCKS blocks per sample write partials (each block a contiguous
// range of the sample's cells, its threads folded in a fixed tree), then one thread per sample folds
// them in block order.
constexpr int STAT_BLOCKS = 256;

__global__ void k_stats_part(Box B, const uint8_t* cell, const float* r, const float* e, float* pm, float* pe) {
  const int s = blockIdx.y, b = blockIdx.x;
  const int per = B.cells();
  const int chunk = (per + STAT_BLOCKS - 1) / STAT_BLOCKS;
  const int c1 = min(per, (b + 1) * chunk);
  float m = 0.f, en = 0.f;
  for (int c = b * chunk + threadIdx.x; c < c1; c += blockDim.x) {
    const int v = s * per + c;
    if ((cell[v] & 3) != FLUID) continue;
    m = fmaxf(m, fabsf(r[v]));
    if (e) en += e[v] * e[v];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    en += __shfl_xor_sync(0xffffffffu, en, o);
  }
  __shared__ float sm[32], se[32];
  if ((threadIdx.x & 31) == 0) {
    sm[threadIdx.x >> 5] = m;
    se[threadIdx.x >> 5] = en;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float a = 0.f, c = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      a = fmaxf(a, sm[w]);
      c += se[w];
    }
    pm[s * STAT_BLOCKS + b] = a;
    pe[s * STAT_BLOCKS + b] = c;
  }
}

__global__ void k_stats_fin(int count, const float* pm, const float* pe, float* scale, float* energy) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= count) return;
  float a = 0.f, c = 0.f;
  for (int b = 0; b < STAT_BLOCKS; b++) {
    a = fmaxf(a, pm[s * STAT_BLOCKS + b]);
    c += pe[s * STAT_BLOCKS + b];
  }
  scale[s] = a > 0.f ? a : 1.f;
  if (energy) energy[s] = c > 0.f ? c : 1.f;
}

// Network input: [r / s, liquid, air, 0 ...] (16 channels).
__global__ void k_pack_input(Box B, const uint8_t* cell, const float* r, const float* scale, bf16* x) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= B.total()) return;
  const int s = v / B.cells();
  const uint8_t t = cell[v] & 3;
  bf16 ch[16];
#pragma unroll
  for (int q = 0; q < 16; q++) ch[q] = __float2bfloat16(0.f);
  if (t == FLUID) ch[0] = __float2bfloat16(r[v] / scale[s]);
  ch[1] = __float2bfloat16(t == FLUID ? 1.f : 0.f);
  ch[2] = __float2bfloat16(t == AIR ? 1.f : 0.f);
  uint4* dst = reinterpret_cast<uint4*>(x + (size_t)v * 16);
  dst[0] = *reinterpret_cast<uint4*>(&ch[0]);
  dst[1] = *reinterpret_cast<uint4*>(&ch[8]);
}

// Output z = s * o[v][0] on liquid cells.
__global__ void k_unpack_output(Box B, const uint8_t* cell, const float* o, const float* scale, float* z) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= B.total()) return;
  const int s = v / B.cells();
  z[v] = (cell[v] & 3) == FLUID ? scale[s] * o[(size_t)v * 16] : 0.f;
}

// Relative squared error per sample, L = mean_s sum_liquid (s o - e)^2 / sum e^2, and its gradient
// with respect to o[v][0] (BF16, 16 channels, the others 0); per-block loss partials.
__global__ void k_loss(Box B, const uint8_t* cell, const float* o, const float* e, const float* scale,
                       const float* energy, bf16* dout, float* loss_part) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (v < B.total()) {
    const int s = v / B.cells();
    float g = 0.f;
    if ((cell[v] & 3) == FLUID) {
      const float diff = scale[s] * o[(size_t)v * 16] - e[v];
      l = diff * diff / (energy[s] * B.count);
      g = 2.f * diff * scale[s] / (energy[s] * B.count);
    }
    bf16 ch[16];
#pragma unroll
    for (int q = 0; q < 16; q++) ch[q] = __float2bfloat16(0.f);
    ch[0] = __float2bfloat16(g);
    uint4* dst = reinterpret_cast<uint4*>(dout + (size_t)v * 16);
    dst[0] = *reinterpret_cast<uint4*>(&ch[0]);
    dst[1] = *reinterpret_cast<uint4*>(&ch[8]);
  }
  __shared__ float sh[256];
  sh[threadIdx.x] = l;
  __syncthreads();
  if (threadIdx.x == 0) {
    float a = 0.f;
    for (int q = 0; q < (int)blockDim.x; q++) a += sh[q];
    loss_part[blockIdx.x] = a;
  }
}

// An unknown of the pressure operator: a liquid cell off the box border.
__device__ __forceinline__ bool is_unknown(const Box& B, const uint8_t* cell, int v, int x, int y, int z) {
  return (cell[v] & 3) == FLUID && x > 0 && y > 0 && z > 0 && x < B.X - 1 && y < B.Y - 1 && z < B.Z - 1;
}

// Energy-norm loss terms, one block per box: d = s o - e on the unknowns, A d and A e with the 7-point
// operator (diagonal: the non-SOLID neighbours, +1 on PL_POISSON_PIN cells; -1 between neighbouring
// unknowns); writes A d, the energy e.Ae and the box's loss term d.Ad / (e.Ae count).
__global__ void k_energy_terms(Box B, const uint8_t* cell, const float* o, const float* e, const float* scale,
                               float* ad, float* energy, float* loss_part) {
  const int s = blockIdx.x;
  const int per = B.cells(), XY = B.X * B.Y;
  const float sc = scale[s];
  double dad = 0, eae = 0;
  for (int c = threadIdx.x; c < per; c += blockDim.x) {
    const int v = s * per + c;
    const int x = c % B.X, y = (c / B.X) % B.Y, z = c / XY;
    if (!is_unknown(B, cell, v, x, y, z)) {
      ad[v] = 0.f;
      continue;
    }
    const int nb6[6] = {v - 1, v + 1, v - B.X, v + B.X, v - XY, v + XY};
    const int nx6[6] = {x - 1, x + 1, x, x, x, x}, ny6[6] = {y, y, y - 1, y + 1, y, y},
              nz6[6] = {z, z, z, z, z - 1, z + 1};
    const float dv = sc * o[(size_t)v * 16] - e[v];
    float diag = (cell[v] & 4) ? 1.f : 0.f;
    float sd = 0.f, se = 0.f;
#pragma unroll
    for (int q = 0; q < 6; q++) {
      const int w = nb6[q];
      if ((cell[w] & 3) != SOLID) diag += 1.f;
      if (is_unknown(B, cell, w, nx6[q], ny6[q], nz6[q])) {
        sd += sc * o[(size_t)w * 16] - e[w];
        se += e[w];
      }
    }
    const float a_d = diag * dv - sd, a_e = diag * e[v] - se;
    ad[v] = a_d;
    dad += double(dv) * a_d;
    eae += double(e[v]) * a_e;
  }
  __shared__ double sh[2][256];
  sh[0][threadIdx.x] = dad;
  sh[1][threadIdx.x] = eae;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int q = 0; q < (int)blockDim.x; q++) {
      a += sh[0][q];
      b += sh[1][q];
    }
    const float en = b > 0 ? float(b) : 1.f;
    energy[s] = en;
    loss_part[s] = float(a) / (en * B.count);
  }
}

// Gradient of the energy-norm loss with respect to o[v][0]: 2 s (A d)_v / (e.Ae count) (A is symmetric).
__global__ void k_energy_grad(Box B, const float* ad, const float* scale, const float* energy, bf16* dout) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= B.total()) return;
  const int s = v / B.cells();
  bf16 ch[16];
#pragma unroll
  for (int q = 0; q < 16; q++) ch[q] = __float2bfloat16(0.f);
  ch[0] = __float2bfloat16(2.f * scale[s] * ad[v] / (energy[s] * B.count));
  uint4* dst = reinterpret_cast<uint4*>(dout + (size_t)v * 16);
  dst[0] = *reinterpret_cast<uint4*>(&ch[0]);
  dst[1] = *reinterpret_cast<uint4*>(&ch[8]);
}

__global__ void k_sum(const float* part, int n, float* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  float a = 0.f;
  for (int i = 0; i < n; i++) a += part[i];
  *out = a;
}

// BF16 weight layouts from the FP32 masters W[t][ci][co]: forward G[t][co][ci] = W[t][ci][co] and
// data-gradient G[t][ci][co] = W[26 - t][ci][co].
__global__ void k_prep_weights(const float* w, int cin, int cout, bf16* gf, bf16* gb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 27 * cin * cout) return;
  const int t = i / (cin * cout), r = i % (cin * cout), ci = r / cout, co = r % cout;
  gf[((size_t)t * cout + co) * cin + ci] = __float2bfloat16(w[i]);
  gb[((size_t)(26 - t) * cin + ci) * cout + co] = __float2bfloat16(w[i]);
}

// Adam (FP32 masters and moments).
__global__ void k_adam(int n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1 - b1) * gi, vi = b2 * v[i] + (1 - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

inline unsigned nb(long long n, int t) { return unsigned((n + t - 1) / t); }

}  // namespace

// ---------------------------------------------------------------- host side

struct UNetImpl {
  // parameters: per layer W[27][cin][cout] then b[cout], contiguous (FP32 masters)
  int off_w[NLAYER], off_b[NLAYER];
  int nparam = 0;
  float *param = nullptr, *grad = nullptr, *m1 = nullptr, *m2 = nullptr;
  bf16 *gf[NLAYER] = {}, *gb[NLAYER] = {};
  void* wmem = nullptr;
  int adam_t = 0;
  // workspace for one box shape and count
  Box b1{}, b2{}, b3{};
  void* ws = nullptr;
  size_t ws_bytes = 0;
  bf16 *x0, *a0, *s1, *p1, *a2, *s2, *p2, *a4, *a5, *c2, *a6, *a7, *c1, *a8, *a9;  // forward
  bf16 *d_o, *d_a9, *d_a8, *d_c1, *d_a7, *d_a6, *d_c2, *d_a5, *d_a4, *d_p2, *d_s2, *d_a2, *d_p1, *d_s1, *d_a0;
  float *o, *scale, *energy, *part, *loss_part, *loss, *ad, *stat_m, *stat_e;
  int nchunk = 0, nloss = 0;
  int loss_kind = 0;  // PL_UNET_LOSS_L2 or PL_UNET_LOSS_ENERGY
  int conv_kernel = PL_UNET_CONV_TCGEN05;  // or PL_UNET_CONV_MMA_SYNC
  int* dev_err = nullptr;  // set by a tcgen05 convolution whose bounded wait gave up

  ~UNetImpl() {
    if (wmem) cudaFree(wmem);
    if (ws) cudaFree(ws);
  }

  int init(uint32_t seed, char* err, size_t errlen) {
    for (int l = 0; l < NLAYER; l++) {
      off_w[l] = nparam;
      nparam += 27 * SPEC[l].cin * SPEC[l].cout;
      off_b[l] = nparam;
      nparam += SPEC[l].cout;
    }
    size_t bf = 0;
    for (int l = 0; l < NLAYER; l++) bf += 2 * size_t(27) * SPEC[l].cin * SPEC[l].cout;
    const size_t total = size_t(nparam) * 4 * 4 + bf * 2 + 4096 + 256;
    if (cudaMalloc(&wmem, total) != cudaSuccess) {
      snprintf(err, errlen, "pl_unet_create: cudaMalloc(%zu) failed", total);
      wmem = nullptr;
      return PL_E_NOMEM;
    }
    cudaMemset(wmem, 0, total);
    char* p = static_cast<char*>(wmem);
    param = (float*)p;
    grad = param + nparam;
    m1 = grad + nparam;
    m2 = m1 + nparam;
    bf16* q = reinterpret_cast<bf16*>(m2 + nparam);
    for (int l = 0; l < NLAYER; l++) {
      gf[l] = q;
      q += size_t(27) * SPEC[l].cin * SPEC[l].cout;
      gb[l] = q;
      q += size_t(27) * SPEC[l].cin * SPEC[l].cout;
    }
    dev_err = reinterpret_cast<int*>(static_cast<char*>(wmem) + total - 256);
    const int big = 227 * 1024;
    cudaFuncSetAttribute(k_conv_tc<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(k_conv_tc<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(k_conv_tc<48>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(k_conv_tc<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(k_conv_tc<96>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(k_conv_tc_row<16, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(k_conv_tc_row<16, 48>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(k_conv_tc_row<48, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    // He initialisation from a fixed generator (mulberry32 + Box-Muller); real input channels only
    std::vector<float> h(nparam, 0.f);
    uint32_t a = seed;
    auto uni = [&]() {
      a += 0x6d2b79f5u;
      uint32_t t = a;
      t = (t ^ (t >> 15)) * (t | 1u);
      t ^= t + (t ^ (t >> 7)) * (t | 61u);
      return (double(t ^ (t >> 14)) + 0.5) / 4294967296.0;
    };
    const int real_in[NLAYER] = {3, 16, 16, 32, 32, 64, 96, 32, 48, 16, 16};
    const int real_out[NLAYER] = {16, 16, 32, 32, 64, 64, 32, 32, 16, 16, 1};
    for (int l = 0; l < NLAYER; l++) {
      const double sd = std::sqrt(2.0 / (27.0 * real_in[l])) * (l == NLAYER - 1 ? 0.1 : 1.0);
      for (int t = 0; t < 27; t++)
        for (int ci = 0; ci < real_in[l]; ci++)
          for (int co = 0; co < real_out[l]; co++) {
            const double u1 = uni(), u2 = uni();
            h[off_w[l] + (t * SPEC[l].cin + ci) * SPEC[l].cout + co] =
                float(sd * std::sqrt(-2.0 * std::log(u1)) * std::cos(2 * PI * u2));
          }
    }
    cudaMemcpy(param, h.data(), size_t(nparam) * 4, cudaMemcpyHostToDevice);
    return cudaGetLastError() == cudaSuccess ? PL_OK : PL_E_CUDA;
  }

  int workspace(int X, int Y, int Z, int count, char* err, size_t errlen) {
    if (ws && b1.X == X && b1.Y == Y && b1.Z == Z && b1.count == count) return PL_OK;
    if (ws) cudaFree(ws);
    ws = nullptr;
    b1 = Box{X, Y, Z, count};
    b2 = Box{X / 2, Y / 2, Z / 2, count};
    b3 = Box{X / 4, Y / 4, Z / 4, count};
    const size_t n1 = size_t(b1.total()), n2 = size_t(b2.total()), n3 = size_t(b3.total());
    nchunk = int((n1 + WG_CHUNK - 1) / WG_CHUNK);
    nloss = int((n1 + 255) / 256);
    size_t maxw = 0;
    for (int l = 0; l < NLAYER; l++) maxw = std::max(maxw, size_t(27) * SPEC[l].cin * SPEC[l].cout);
    std::vector<size_t> sz = {
        n1 * 16, n1 * 16, n1 * 16, n2 * 16, n2 * 32, n2 * 32, n3 * 32, n3 * 64, n3 * 64, n2 * 96, n2 * 32, n2 * 32,
        n1 * 48, n1 * 16, n1 * 16,                                                               // forward (bf16 elems)
        n1 * 16, n1 * 16, n1 * 16, n1 * 48, n2 * 32, n2 * 32, n2 * 96, n3 * 64, n3 * 64, n3 * 32, n2 * 32, n2 * 32,
        n2 * 16, n1 * 16, n1 * 16};                                                              // gradients
    size_t bytes = 0;
    for (size_t s : sz) bytes += ((s * 2 + 255) & ~size_t(255));
    const size_t fbytes = n1 * 16 * 4 + 2 * size_t(count) * 4 + size_t(nchunk) * maxw * 4 + size_t(nloss) * 4 + 1024 +
                          n1 * 4 + 256 + 2 * size_t(count) * STAT_BLOCKS * 4 + 256;
    if (cudaMalloc(&ws, bytes + fbytes + 4096) != cudaSuccess) {
      ws = nullptr;
      snprintf(err, errlen, "pl_unet: workspace cudaMalloc(%zu) failed", bytes + fbytes);
      return PL_E_NOMEM;
    }
    ws_bytes = bytes + fbytes;
    char* p = static_cast<char*>(ws);
    std::vector<bf16*> ptr;
    for (size_t s : sz) {
      ptr.push_back((bf16*)p);
      p += (s * 2 + 255) & ~size_t(255);
    }
    bf16** fw[] = {&x0, &a0, &s1, &p1, &a2, &s2, &p2, &a4, &a5, &c2, &a6, &a7, &c1, &a8, &a9,
                   &d_o, &d_a9, &d_a8, &d_c1, &d_a7, &d_a6, &d_c2, &d_a5, &d_a4, &d_p2, &d_s2, &d_a2, &d_p1, &d_s1, &d_a0};
    for (size_t i = 0; i < ptr.size(); i++) *fw[i] = ptr[i];
    o = (float*)p;
    p += n1 * 16 * 4;
    scale = (float*)p;
    p += size_t(count) * 4;
    energy = (float*)p;
    p += size_t(count) * 4;
    p = (char*)(((uintptr_t)p + 255) & ~uintptr_t(255));
    part = (float*)p;
    p += size_t(nchunk) * maxw * 4;
    loss_part = (float*)p;
    p += size_t(nloss) * 4;
    loss = (float*)p;
    p += 1024;
    ad = (float*)p;
    p += n1 * 4;
    p = (char*)(((uintptr_t)p + 255) & ~uintptr_t(255));
    stat_m = (float*)p;
    stat_e = stat_m + size_t(count) * STAT_BLOCKS;
    return PL_OK;
  }

  void prep_weights(cudaStream_t st) {
    for (int l = 0; l < NLAYER; l++) {
      const int n = 27 * SPEC[l].cin * SPEC[l].cout;
      k_prep_weights<<<nb(n, 256), 256, 0, st>>>(param + off_w[l], SPEC[l].cin, SPEC[l].cout, gf[l], gb[l]);
    }
  }

  // out = conv_l(in) (forward, G = gf) or the data gradient (G = gb; then nout = cin of the layer).
  void conv(const Box& B, const bf16* in, int cin, const bf16* G, int nout, const float* bias, int relu,
            const bf16* mask, bf16* out_bf, float* out_f32, cudaStream_t st) {
    if (conv_kernel == PL_UNET_CONV_TCGEN05 && B.X % 128 == 0 &&
        ((cin == 16 && (nout == 16 || nout == 48)) || (cin == 48 && nout == 16))) {
      // the full-resolution convolutions (and their data gradients) of boxes 128 or 256 wide
      const unsigned blocks = tc_row_blocks(B);
      const size_t sm = tc_row_smem(cin, nout);
      if (cin == 16 && nout == 16)
        k_conv_tc_row<16, 16><<<blocks, 128, sm, st>>>(B, in, cin, G, bias, relu, mask, out_bf, out_f32, dev_err);
      else if (cin == 16)
        k_conv_tc_row<16, 48><<<blocks, 128, sm, st>>>(B, in, cin, G, bias, relu, mask, out_bf, out_f32, dev_err);
      else
        k_conv_tc_row<48, 16><<<blocks, 128, sm, st>>>(B, in, cin, G, bias, relu, mask, out_bf, out_f32, dev_err);
      return;
    }
    if (conv_kernel == PL_UNET_CONV_TCGEN05) {
      const unsigned blocks = nb(B.total(), 128);
      const size_t sm = tc_smem(cin, nout);
      if (nout == 16)
        k_conv_tc<16><<<blocks, 128, sm, st>>>(B, in, cin, G, bias, relu, mask, out_bf, out_f32, dev_err);
      else if (nout == 32)
        k_conv_tc<32><<<blocks, 128, sm, st>>>(B, in, cin, G, bias, relu, mask, out_bf, out_f32, dev_err);
      else if (nout == 48)
        k_conv_tc<48><<<blocks, 128, sm, st>>>(B, in, cin, G, bias, relu, mask, out_bf, out_f32, dev_err);
      else if (nout == 64)
        k_conv_tc<64><<<blocks, 128, sm, st>>>(B, in, cin, G, bias, relu, mask, out_bf, out_f32, dev_err);
      else
        k_conv_tc<96><<<blocks, 128, sm, st>>>(B, in, cin, G, bias, relu, mask, out_bf, out_f32, dev_err);
      return;
    }
    const long long warps = (B.total() + 15) / 16;
    const unsigned blocks = nb(warps * 32, 128);
    if (nout == 16)
      k_conv<16><<<blocks, 128, 0, st>>>(B, in, cin, G, bias, relu, mask, out_bf, out_f32);
    else if (nout == 32)
      k_conv<32><<<blocks, 128, 0, st>>>(B, in, cin, G, bias, relu, mask, out_bf, out_f32);
    else if (nout == 48)
      k_conv<48><<<blocks, 128, 0, st>>>(B, in, cin, G, bias, relu, mask, out_bf, out_f32);
    else if (nout == 64)
      k_conv<64><<<blocks, 128, 0, st>>>(B, in, cin, G, bias, relu, mask, out_bf, out_f32);
    else
      k_conv<96><<<blocks, 128, 0, st>>>(B, in, cin, G, bias, relu, mask, out_bf, out_f32);
  }

  void forward(const uint8_t* cell, const float* r, cudaStream_t st) {
    prep_weights(st);
    k_stats_part<<<dim3(STAT_BLOCKS, b1.count), 256, 0, st>>>(b1, cell, r, nullptr, stat_m, stat_e);
    k_stats_fin<<<nb(b1.count, 128), 128, 0, st>>>(b1.count, stat_m, stat_e, scale, nullptr);
    k_pack_input<<<nb(b1.total(), 256), 256, 0, st>>>(b1, cell, r, scale, x0);
    auto L = [&](int l, const Box& B, const bf16* in, bf16* out, int relu, float* f32) {
      conv(B, in, SPEC[l].cin, gf[l], SPEC[l].cout, param + off_b[l], relu, nullptr, out, f32, st);
    };
    L(0, b1, x0, a0, 1, nullptr);
    L(1, b1, a0, s1, 1, nullptr);
    k_pool<<<nb((long long)b2.total() * 16, 256), 256, 0, st>>>(b1, b2, s1, 16, p1);
    L(2, b2, p1, a2, 1, nullptr);
    L(3, b2, a2, s2, 1, nullptr);
    k_pool<<<nb((long long)b3.total() * 32, 256), 256, 0, st>>>(b2, b3, s2, 32, p2);
    L(4, b3, p2, a4, 1, nullptr);
    L(5, b3, a4, a5, 1, nullptr);
    k_up_concat<<<nb((long long)b2.total() * 96 / 8, 256), 256, 0, st>>>(b2, b3, a5, 64, s2, 32, c2);
    L(6, b2, c2, a6, 1, nullptr);
    L(7, b2, a6, a7, 1, nullptr);
    k_up_concat<<<nb((long long)b1.total() * 48 / 8, 256), 256, 0, st>>>(b1, b2, a7, 32, s1, 16, c1);
    L(8, b1, c1, a8, 1, nullptr);
    L(9, b1, a8, a9, 1, nullptr);
    L(10, b1, a9, nullptr, 0, o);
  }

  // Weight and bias gradient of layer l from its input and the gradient of its pre-activation.
  void wgrad(int l, const Box& B, const bf16* in, const bf16* d, cudaStream_t st) {
    const int ci = SPEC[l].cin, co = SPEC[l].cout;
    const int nch = (B.total() + WG_CHUNK - 1) / WG_CHUNK;
    dim3 grid(nch, 27);
#define WG(CI, CO) \
  if (ci == CI && co == CO) k_wgrad<CI, CO><<<grid, 128, 0, st>>>(B, in, d, part);
    WG(16, 16) WG(16, 32) WG(32, 32) WG(32, 64) WG(64, 64) WG(96, 32) WG(48, 16)
#undef WG
    const int n = 27 * ci * co;
    k_wgrad_reduce<<<nb(n, 256), 256, 0, st>>>(part, nch, n, grad + off_w[l]);
    k_bgrad_part<<<nch, (256 / co) * co, 0, st>>>(B, d, co, part);
    k_wgrad_reduce<<<1, 256, 0, st>>>(part, nch, co, grad + off_b[l]);
  }

  // Data gradient through layer l: din = conv^T(d) masked by the ReLU of mask (null: no mask).
  void dgrad(int l, const Box& B, const bf16* d, const bf16* mask, bf16* din, cudaStream_t st) {
    conv(B, d, SPEC[l].cout, gb[l], SPEC[l].cin, nullptr, 0, mask, din, nullptr, st);
  }

  void backward(cudaStream_t st) {
    // d_o holds dL/do (channel 0); ReLU-free output layer
    wgrad(10, b1, a9, d_o, st);
    dgrad(10, b1, d_o, a9, d_a9, st);
    wgrad(9, b1, a8, d_a9, st);
    dgrad(9, b1, d_a9, a8, d_a8, st);
    wgrad(8, b1, c1, d_a8, st);
    dgrad(8, b1, d_a8, nullptr, d_c1, st);
    k_up_concat_bwd_coarse<<<nb((long long)b2.total() * 32, 256), 256, 0, st>>>(b1, b2, d_c1, 32, 48, a7, d_a7);
    k_concat_bwd_skip<<<nb((long long)b1.total() * 16, 256), 256, 0, st>>>(b1.total(), d_c1, 32, 48, 16, d_s1);
    wgrad(7, b2, a6, d_a7, st);
    dgrad(7, b2, d_a7, a6, d_a6, st);
    wgrad(6, b2, c2, d_a6, st);
    dgrad(6, b2, d_a6, nullptr, d_c2, st);
    k_up_concat_bwd_coarse<<<nb((long long)b3.total() * 64, 256), 256, 0, st>>>(b2, b3, d_c2, 64, 96, a5, d_a5);
    k_concat_bwd_skip<<<nb((long long)b2.total() * 32, 256), 256, 0, st>>>(b2.total(), d_c2, 64, 96, 32, d_s2);
    wgrad(5, b3, a4, d_a5, st);
    dgrad(5, b3, d_a5, a4, d_a4, st);
    wgrad(4, b3, p2, d_a4, st);
    dgrad(4, b3, d_a4, nullptr, d_p2, st);
    k_pool_bwd_add<<<nb((long long)b2.total() * 32, 256), 256, 0, st>>>(b2, b3, d_p2, 32, d_s2);
    k_relu_mask<<<nb((long long)b2.total() * 32, 256), 256, 0, st>>>(b2.total() * 32, d_s2, s2);
    wgrad(3, b2, a2, d_s2, st);
    dgrad(3, b2, d_s2, a2, d_a2, st);
    wgrad(2, b2, p1, d_a2, st);
    dgrad(2, b2, d_a2, nullptr, d_p1, st);
    k_pool_bwd_add<<<nb((long long)b1.total() * 16, 256), 256, 0, st>>>(b1, b2, d_p1, 16, d_s1);
    k_relu_mask<<<nb((long long)b1.total() * 16, 256), 256, 0, st>>>(b1.total() * 16, d_s1, s1);
    wgrad(1, b1, a0, d_s1, st);
    dgrad(1, b1, d_s1, a0, d_a0, st);
    wgrad(0, b1, x0, d_a0, st);
  }

  void loss_and_grad(const uint8_t* cell, const float* e, cudaStream_t st) {
    if (loss_kind == PL_UNET_LOSS_ENERGY) {
      k_energy_terms<<<b1.count, 256, 0, st>>>(b1, cell, o, e, scale, ad, energy, loss_part);
      k_energy_grad<<<nb(b1.total(), 256), 256, 0, st>>>(b1, ad, scale, energy, d_o);
      k_sum<<<1, 32, 0, st>>>(loss_part, b1.count, loss);
      return;
    }
    k_stats_part<<<dim3(STAT_BLOCKS, b1.count), 256, 0, st>>>(b1, cell, e, e, stat_m, stat_e);  // target energy
    k_stats_fin<<<nb(b1.count, 128), 128, 0, st>>>(b1.count, stat_m, stat_e, part, energy);
    k_loss<<<nb(b1.total(), 256), 256, 0, st>>>(b1, cell, o, e, scale, energy, d_o, loss_part);
    k_sum<<<1, 32, 0, st>>>(loss_part, nloss, loss);
  }
};

namespace {
int check_box(int X, int Y, int Z, int count, char* err, size_t errlen) {
  if (X < 4 || Y < 4 || Z < 4 || X % 4 || Y % 4 || Z % 4 || count < 1 ||
      (long long)X * Y * Z * count > (1ll << 26)) {
    snprintf(err, errlen, "pl_unet: box %dx%dx%d x %d must be multiples of 4 with at most 2^26 cells", X, Y, Z,
             count);
    return PL_E_ARG;
  }
  return PL_OK;
}
}  // namespace

UNetImpl* unet_create(uint32_t seed, char* err, size_t errlen, int* rc) {
  UNetImpl* u = new UNetImpl();
  *rc = u->init(seed, err, errlen);
  if (*rc) {
    delete u;
    return nullptr;
  }
  return u;
}

void unet_destroy(UNetImpl* u) { delete u; }

int unet_nparams(const UNetImpl* u) { return u->nparam; }

void unet_set_loss(UNetImpl* u, int kind) { u->loss_kind = kind; }

int unet_get_params(UNetImpl* u, float* host) {
  return cudaMemcpy(host, u->param, size_t(u->nparam) * 4, cudaMemcpyDeviceToHost) == cudaSuccess ? PL_OK
                                                                                                   : PL_E_CUDA;
}

int unet_set_params(UNetImpl* u, const float* host) {
  u->adam_t = 0;
  cudaMemset(u->m1, 0, size_t(u->nparam) * 4);
  cudaMemset(u->m2, 0, size_t(u->nparam) * 4);
  return cudaMemcpy(u->param, host, size_t(u->nparam) * 4, cudaMemcpyHostToDevice) == cudaSuccess ? PL_OK
                                                                                                   : PL_E_CUDA;
}

int unet_prepare(UNetImpl* u, int X, int Y, int Z, int count, char* err, size_t errlen) {
  int rc = check_box(X, Y, Z, count, err, errlen);
  return rc ? rc : u->workspace(X, Y, Z, count, err, errlen);
}

int unet_apply(UNetImpl* u, const uint8_t* cell, const float* r, float* z, int X, int Y, int Z, int count,
               cudaStream_t st, char* err, size_t errlen) {
  int rc = check_box(X, Y, Z, count, err, errlen);
  if (!rc) rc = u->workspace(X, Y, Z, count, err, errlen);
  if (rc) return rc;
  u->forward(cell, r, st);
  k_unpack_output<<<nb(u->b1.total(), 256), 256, 0, st>>>(u->b1, cell, u->o, u->scale, z);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    snprintf(err, errlen, "pl_unet_apply: %s", cudaGetErrorString(e));
    return PL_E_CUDA;
  }
  return PL_OK;
}

int unet_gradient(UNetImpl* u, const uint8_t* cell, const float* r, const float* e, int X, int Y, int Z, int count,
                  float lr, int update, float* loss, float* grad_host, cudaStream_t st, char* err, size_t errlen) {
  int rc = check_box(X, Y, Z, count, err, errlen);
  if (!rc) rc = u->workspace(X, Y, Z, count, err, errlen);
  if (rc) return rc;
  u->forward(cell, r, st);
  u->loss_and_grad(cell, e, st);
  u->backward(st);
  if (update) {
    u->adam_t++;
    const float b1 = 0.9f, b2 = 0.999f;
    k_adam<<<nb(u->nparam, 256), 256, 0, st>>>(u->nparam, u->param, u->grad, u->m1, u->m2, lr, b1, b2, 1e-8f,
                                               1.f - std::pow(b1, float(u->adam_t)),
                                               1.f - std::pow(b2, float(u->adam_t)));
  }
  int tc_err = 0;
  cudaError_t ce = cudaMemcpyAsync(loss, u->loss, 4, cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(&tc_err, u->dev_err, 4, cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess && grad_host)
    ce = cudaMemcpyAsync(grad_host, u->grad, size_t(u->nparam) * 4, cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  if (ce != cudaSuccess) {
    snprintf(err, errlen, "pl_unet: %s", cudaGetErrorString(ce));
    return PL_E_CUDA;
  }
  if (tc_err) {
    snprintf(err, errlen, "pl_unet: a tensor-core convolution's bounded wait gave up");
    return PL_E_TIMEOUT;
  }
  return PL_OK;
}

int unet_set_conv_kernel(UNetImpl* u, int kind) {
  if (kind != PL_UNET_CONV_TCGEN05 && kind != PL_UNET_CONV_MMA_SYNC) return PL_E_ARG;
  u->conv_kernel = kind;
  return PL_OK;
}

int unet_error(UNetImpl* u) {
  int e = 0;
  cudaMemcpy(&e, u->dev_err, 4, cudaMemcpyDeviceToHost);
  return e;
}

}  // namespace pl
