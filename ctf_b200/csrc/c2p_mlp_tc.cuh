// Learned c2p guess on the 5th-generation tensor cores (tcgen05), 128 zones per CTA.
//
// Each CTA of 128 threads evaluates the network for 128 rows at once: M = 128 maps row m to
// TMEM lane m and to thread m.  Operands are BF16 in shared memory in the canonical K-major,
// no-swizzle layout (8-row x 16-byte core matrices: element (r, k) of an R x K operand at
// ((r/8)*(K/8) + k/8)*128 + (r%8)*16 + (k%8)*2 bytes; LBO = 128 B between K-adjacent core
// matrices, SBO = K*16 B between row groups).  Accumulators are FP32 in TMEM (64 columns);
// each layer's epilogue reads its row with tcgen05.ld (32x32b), adds the bias, applies tanh
// (packed BF16 pairs) and writes the next layer's BF16 operand.  One thread issues the MMAs
// and commits them to an
// mbarrier; every wait on it is bounded and reports a timeout instead of hanging.
//
// Network image on the device (bytes, built by mgpu_set_c2p_network from the FP32 weights):
//   [0, 2048)       W1  64 x 16 (inputs 0..4, zero padded)
//   [2048, 10240)   W2  64 x 64
//   [10240, 18432)  W3  64 x 64
//   [18432, 20480)  W4  16 x 64 (rows 0, 1; zero padded)
//   [20480, 21312)  float b1[64] b2[64] b3[64] b4[2] xmean[5] xstd[5] ymean[2] ystd[2]
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>
#include "c2p_mlp_net.cuh"

namespace mgpu {
namespace tc {

constexpr int W1_OFF = 0, W2_OFF = 2048, W3_OFF = 10240, W4_OFF = 18432, F_OFF = 20480;
constexpr int F_B1 = 0, F_B2 = 64, F_B3 = 128, F_B4 = 192, F_XM = 194, F_XS = 199, F_YM = 204, F_YS = 206;
constexpr int IMAGE_BYTES = F_OFF + 208 * 4;                 // 21312
constexpr int A_BYTES = 128 * 64 * 2;                        // activation operand, 16 KB
constexpr int IMAGE_SLOT = (IMAGE_BYTES + 1023) / 1024 * 1024;
constexpr int SMEM_BYTES = 1024 + IMAGE_SLOT + A_BYTES + 64;   // alignment slack, image, A, mbarrier + TMEM slot
constexpr int TMEM_COLS = 64;
constexpr unsigned WAIT_LIMIT = 1u << 22;                    // bounded mbarrier polls

__host__ __device__ constexpr int canon_offset(int r, int k, int K)
{
  return ((r / 8) * (K / 8) + k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t) __cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
  uint64_t d = 0;
  d |= (uint64_t) ((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t) ((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t) ((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t) 1 << 46;   // descriptor version for sm_100; base offset 0, no swizzle
  return d;
}

// kind::f16 instruction descriptor: F32 accumulate, BF16 A and B, both K-major, M = 128.
__device__ __forceinline__ uint32_t idesc_bf16(int N)
{
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t) (N >> 3) << 17) | ((uint32_t) (128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

// Bounded wait on an mbarrier phase; returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase)
{
  for (unsigned i = 0; i < WAIT_LIMIT; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v)
{
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Two floats -> packed BF16 pair (a in the low half), one paired conversion instruction.
__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b)
{
  const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&v);
}

// Stores 8 consecutive K values of row r (K-chunk c) of an operand with K columns.
__device__ __forceinline__ void store_chunk(unsigned char *A, int r, int c, int K, const float *v)
{
  uint4 q;
  q.x = pack_bf16x2(v[0], v[1]);
  q.y = pack_bf16x2(v[2], v[3]);
  q.z = pack_bf16x2(v[4], v[5]);
  q.w = pack_bf16x2(v[6], v[7]);
  *reinterpret_cast<uint4 *>(A + canon_offset(r, 8 * c, K)) = q;
}

// tanh of two packed BF16 values (the PTX tanh.approx.bf16x2 instruction): the activations
// are BF16 operands of the next layer anyway, so the activation is evaluated at that width.
__device__ __forceinline__ uint32_t tanh_bf16x2(uint32_t x)
{
  uint32_t y;
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(y) : "r"(x));
  return y;
}

// CTA-wide network evaluation context (one per CTA; all 128 threads call every method).
struct TcNet {
  unsigned char *img;   // network image in shared memory
  unsigned char *A;     // activation operand
  uint32_t mbar;        // shared address of the mbarrier
  uint32_t tmem;        // TMEM base (lane 0, column 0)
  uint32_t phase;
  int ok;               // 0 after a timed-out wait: the CTA stops using the tensor cores

  // One layer: D[128 x N] = A[128 x K] * W^T, K in steps of 16, then wait for it.
  __device__ __forceinline__ bool layer(uint32_t w_addr, int K, int N)
  {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (threadIdx.x == 0) {
      const uint32_t a_addr = smem_u32(A);
      const uint32_t id = idesc_bf16(N);
      for (int s = 0; s < K / 16; ++s)
        mma_bf16(tmem, sdesc(a_addr + 256 * s, 128, K * 16), sdesc(w_addr + 256 * s, 128, K * 16), id, s > 0);
      mma_commit(mbar);
    }
    const bool done = mbar_wait(mbar, phase);
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    return __syncthreads_and(done) != 0;
  }

  // Epilogue of a hidden layer: this thread's row of D (+bias, tanh) -> BF16 row of A (K = 64).
  __device__ __forceinline__ void hidden_epilogue(const float *bias)
  {
    const int r = threadIdx.x, warp = r >> 5;
    const uint32_t row = tmem + ((uint32_t) (warp * 32) << 16);
#pragma unroll 1
    for (int c0 = 0; c0 < 64; c0 += 16) {
      float v[16];
      tmem_ld16(row + (uint32_t) c0, v);
      uint32_t h[8];
#pragma unroll
      for (int i = 0; i < 8; ++i)
        h[i] = tanh_bf16x2(pack_bf16x2(v[2 * i] + bias[c0 + 2 * i], v[2 * i + 1] + bias[c0 + 2 * i + 1]));
      *reinterpret_cast<uint4 *>(A + canon_offset(r, c0, 64)) = make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4 *>(A + canon_offset(r, c0 + 8, 64)) = make_uint4(h[4], h[5], h[6], h[7]);
    }
  }

  // Full forward pass for this thread's (normalised) feature row; false if the CTA has
  // stopped using the tensor cores.
  __device__ __forceinline__ bool forward(const float *xn, float *y)
  {
    const float *f = reinterpret_cast<const float *>(img + F_OFF);
    {
      float v[8] = {xn[0], xn[1], xn[2], xn[3], xn[4], 0.f, 0.f, 0.f};
      const float z[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      store_chunk(A, threadIdx.x, 0, 16, v);
      store_chunk(A, threadIdx.x, 1, 16, z);
    }
    const uint32_t w = smem_u32(img);
    if (!ok || !layer(w + W1_OFF, 16, 64)) { ok = 0; return false; }
    hidden_epilogue(f + F_B1);
    if (!layer(w + W2_OFF, 64, 64)) { ok = 0; return false; }
    hidden_epilogue(f + F_B2);
    if (!layer(w + W3_OFF, 64, 64)) { ok = 0; return false; }
    hidden_epilogue(f + F_B3);
    if (!layer(w + W4_OFF, 64, 16)) { ok = 0; return false; }
    float v[16];
    tmem_ld16(tmem + ((uint32_t) ((threadIdx.x >> 5) * 32) << 16), v);
    y[0] = (v[0] + f[F_B4 + 0]) * f[F_YS + 0] + f[F_YM + 0];
    y[1] = (v[1] + f[F_B4 + 1]) * f[F_YS + 1] + f[F_YM + 1];
    // every thread's TMEM reads complete before the next tile's first MMA overwrites it
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    return true;
  }

  __device__ __forceinline__ void normalise(const float *x, float *xn) const
  {
    const float *f = reinterpret_cast<const float *>(img + F_OFF);
#pragma unroll
    for (int i = 0; i < 5; ++i) xn[i] = (x[i] - f[F_XM + i]) / f[F_XS + i];
  }
};

// Set-up: copy the network image to shared memory, allocate TMEM, initialise the mbarrier.
// `smem` is the CTA's dynamic shared memory (SMEM_BYTES).
__device__ __forceinline__ TcNet tc_setup(unsigned char *smem, const unsigned char *image)
{
  TcNet n;
  unsigned char *base = (unsigned char *) (((uintptr_t) smem + 1023) & ~(uintptr_t) 1023);
  n.img = base;
  n.A = base + IMAGE_SLOT;
  uint64_t *bar = reinterpret_cast<uint64_t *>(n.A + A_BYTES);
  uint32_t *slot = reinterpret_cast<uint32_t *>(bar + 1);
  for (int i = threadIdx.x; i < IMAGE_BYTES / 16; i += blockDim.x)
    reinterpret_cast<uint4 *>(n.img)[i] = reinterpret_cast<const uint4 *>(image)[i];
  n.mbar = smem_u32(bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(n.mbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  n.tmem = *slot;
  n.phase = 0;
  n.ok = 1;
  return n;
}

// Release TMEM (warp 0, the warp that allocated it); all threads of the CTA must call.  After
// a timed-out wait, first wait once more (bounded) for the MMAs still in flight.
__device__ __forceinline__ void tc_teardown(TcNet &n)
{
  if (!n.ok) mbar_wait(n.mbar, n.phase ^ 1u);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (threadIdx.x < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(n.tmem), "r"(TMEM_COLS) : "memory");
}

}  // namespace tc
}  // namespace mgpu
