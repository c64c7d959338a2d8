// dnl_mlp.cuh - the learned Newton initial guess of the radial return: a
// 5 -> 64 -> 64 -> 64 -> 1 SiLU network whose three hidden layers run on the
// 5th-generation tensor cores (tcgen05.mma, BF16 operands in shared memory,
// FP32 accumulators in tensor memory) over a tile of TILE = 128 Gauss points,
// one row per thread, and whose output layer is an FP32 dot product.
//
// Included by dnl_kernels.cuh after the bulk-copy / mbarrier primitives.
//
// Operand layout ("K-major, no swizzle" canonical layout of the UMMA shared
// memory descriptor): an R x K BF16 matrix is stored as K/8 column chunks of
// R rows x 16 bytes; inside a chunk, 8-row core matrices of 128 contiguous
// bytes.  Element (r, k) sits at byte
//     (k / 8) * (R * 16) + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,
// the leading byte offset (between the two 8-wide K chunks of one K = 16
// instruction) is R * 16 and the stride byte offset (between 8-row groups) is 128.
#pragma once

namespace mlp
{
constexpr int NIN = 5;    // trial sigma_eq / A, eps_p, log(1 + rate / rate0), T / Tm, log(3 G dt rate0 / A)
constexpr int KIN = 16;   // input width padded to one K = 16 instruction
constexpr int H = 64;     // hidden width
constexpr int M = TILE;   // rows per tile (one per thread)

// device image of the network (global memory, copied to shared memory as is)
constexpr uint32_t OFF_W1 = 0;                    // H x KIN bf16, canonical
constexpr uint32_t OFF_W2 = OFF_W1 + H * KIN * 2; // H x H bf16
constexpr uint32_t OFF_W3 = OFF_W2 + H * H * 2;
constexpr uint32_t OFF_B1 = OFF_W3 + H * H * 2;   // fp32 biases
constexpr uint32_t OFF_B2 = OFF_B1 + H * 4;
constexpr uint32_t OFF_B3 = OFF_B2 + H * 4;
constexpr uint32_t OFF_W4 = OFF_B3 + H * 4;       // fp32 output weights
constexpr uint32_t OFF_MISC = OFF_W4 + H * 4;     // b4, in_mean[5], in_scale[5], out_exp, in_clip, pad
constexpr uint32_t IMAGE_BYTES = OFF_MISC + 16 * 4;
// training adds the transposed hidden weights (for dh = dz W), after the image
constexpr uint32_t OFF_W2T = 0, OFF_W3T = H * H * 2, TRANS_BYTES = 2 * H * H * 2;
// activation tile (M x H bf16), after the image in shared memory
constexpr uint32_t OFF_ACT = (IMAGE_BYTES + 255) & ~255u;
constexpr uint32_t ACT_BYTES = M * H * 2;
constexpr uint32_t SMEM_BYTES = OFF_ACT + ACT_BYTES;
constexpr uint32_t TMEM_COLS = 64;
static_assert(IMAGE_BYTES % 16 == 0, "bulk copies move multiples of 16 bytes");
static_assert(M == 128, "one tcgen05 M = 128 tile per block");

__host__ __device__ constexpr uint32_t canon(int r, int k, int R)
{
  return (uint32_t)((k >> 3) * (R * 16) + (r >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// UMMA shared memory descriptor, no swizzle (layout type 0), descriptor version 1
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: D fp32 (bit 4), A and B bf16 (bits 7, 10),
// both K-major, N >> 3 at bit 17, M >> 4 at bit 24
template <int MM, int NN> __host__ __device__ constexpr uint32_t idesc_bf16()
{
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NN >> 3) << 17) | ((uint32_t)(MM >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
  asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
               " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
               "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
               : "memory");
}

// completion of the MMAs issued so far by this thread, as one arrival on `bar`
__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void block_bar() { asm volatile("bar.sync 1, %0;" ::"n"(TILE) : "memory"); }

// 16 consecutive fp32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
  uint32_t r[16];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                 "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                 "=r"(r[15])
               : "r"(taddr)
               : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++)
    v[i] = __uint_as_float(r[i]);
}

// Tensor-memory allocation of one block (warp 0 allocates and frees).
__device__ __forceinline__ void tmem_alloc(uint32_t *slot)
{
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
               "n"(TMEM_COLS)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr)
{
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "n"(TMEM_COLS) : "memory");
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z)
{
  const float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// Input features of one Gauss point from its trial state (the same function
// feeds the harvested training pairs and the guess).
__device__ __forceinline__ void features(float Strial, float epsp, float depsp, float T, float twoG, float dt,
                                         const MatDev &mp, float (&x)[NIN])
{
  const float A = (float)mp.A;
  x[0] = Strial / A;
  x[1] = epsp;
  x[2] = log1pf(depsp / (float)mp.depsp0);
  x[3] = T / (float)mp.Tm;
  x[4] = __logf(1.5f * twoG * dt * (float)mp.depsp0 / A);
}

// One block's view of the network in shared memory: the image, the
// activation tile, the accumulator columns in tensor memory and the mbarrier
// the MMAs complete on.  Every thread of the block calls forward() at the
// same point of a convergent path.
struct Tile
{
  unsigned char *smem; // 1024-aligned: image at 0
  uint32_t act;        // offset of the activation tile (the A operand)
  uint32_t tmem;       // base address of TMEM_COLS columns
  uint64_t *bar;
  uint32_t phase;
  int *err;
  bool broken; // a wait gave up: no further tensor-core work in this block

  __device__ __forceinline__ bool wait()
  {
    if (broken)
      return false;
    const bool ok = mbar_wait(bar, phase);
    phase ^= 1;
    if (!ok)
    {
      atomicExch(err, 2);
      broken = true;
    }
    fence_after_sync();
    return ok;
  }

  // issue one layer (thread 0): D[M x H] = A[M x K] . W[H x K]^T over K / 16 steps
  __device__ __forceinline__ void layer(uint32_t a_off, uint32_t w_off, int K)
  {
    const uint32_t sa = smem_u32(smem + a_off), sw = smem_u32(smem + w_off);
    constexpr uint32_t idesc = idesc_bf16<M, H>();
    for (int s = 0; s < K / 16; s++)
      mma_bf16(tmem, sdesc(sa + s * 2 * (M * 16), M * 16, 128), sdesc(sw + s * 2 * (H * 16), H * 16, 128), idesc,
               s > 0 ? 1u : 0u);
    mma_commit(bar);
  }

  // write this thread's row of the next A operand (bf16) from 64 fp32 values
  __device__ __forceinline__ void put_row(int t, const float (&h)[H])
  {
#pragma unroll
    for (int c = 0; c < H / 8; c++)
    {
      uint4 v;
      __nv_bfloat162 p0 = __floats2bfloat162_rn(h[8 * c], h[8 * c + 1]);
      __nv_bfloat162 p1 = __floats2bfloat162_rn(h[8 * c + 2], h[8 * c + 3]);
      __nv_bfloat162 p2 = __floats2bfloat162_rn(h[8 * c + 4], h[8 * c + 5]);
      __nv_bfloat162 p3 = __floats2bfloat162_rn(h[8 * c + 6], h[8 * c + 7]);
      v.x = *reinterpret_cast<uint32_t *>(&p0);
      v.y = *reinterpret_cast<uint32_t *>(&p1);
      v.z = *reinterpret_cast<uint32_t *>(&p2);
      v.w = *reinterpret_cast<uint32_t *>(&p3);
      *reinterpret_cast<uint4 *>(smem + act + canon(t, 8 * c, M)) = v;
    }
  }

  // hand the freshly written A operand to the tensor cores and run one layer
  __device__ __forceinline__ void run_layer(int t, uint32_t w_off, int K)
  {
    fence_async_smem();
    fence_before_sync();
    block_bar();
    fence_after_sync();
    if (t == 0 && !broken)
      layer(act, w_off, K);
    wait();
  }

  // the normalised, zero-padded input row as the first A operand
  __device__ __forceinline__ void put_input(int t, const float (&x)[NIN], float (&xin)[KIN])
  {
    const float *misc = reinterpret_cast<const float *>(smem + OFF_MISC);
    const float clip = misc[12];
#pragma unroll
    for (int i = 0; i < KIN; i++)
    {
      float v = (i < NIN) ? (x[i] - misc[1 + i]) * misc[6 + i] : 0.0f;
      if (clip > 0.0f)
        v = fminf(fmaxf(v, -clip), clip);
      xin[i] = v;
    }
    uint4 v[2];
    uint32_t *w = reinterpret_cast<uint32_t *>(v);
#pragma unroll
    for (int i = 0; i < KIN / 2; i++)
    {
      __nv_bfloat162 p = __floats2bfloat162_rn(xin[2 * i], xin[2 * i + 1]);
      w[i] = *reinterpret_cast<uint32_t *>(&p);
    }
    *reinterpret_cast<uint4 *>(smem + act + canon(t, 0, M)) = v[0];
    *reinterpret_cast<uint4 *>(smem + act + canon(t, 8, M)) = v[1];
  }

  // z = accumulator row + bias (pre-activations of this thread's row)
  __device__ __forceinline__ void read_row(const float *bias, float (&z)[H])
  {
    const uint32_t lane_base = (uint32_t)(threadIdx.x & ~31) << 16;
#pragma unroll
    for (int c = 0; c < H / 16; c++)
    {
      float v[16];
      tmem_ld16(tmem + lane_base + 16 * c, v);
#pragma unroll
      for (int i = 0; i < 16; i++)
        z[16 * c + i] = v[i] + bias[16 * c + i];
    }
  }

  // Forward pass of the block's tile; x holds this thread's raw features
  // (zeros for a row without a plastic trial).  Returns the output of the row.
  __device__ __forceinline__ float forward(int t, const float (&x)[NIN])
  {
    const float *misc = reinterpret_cast<const float *>(smem + OFF_MISC);
    {
      float xin[KIN];
      put_input(t, x, xin);
    }
    float z[H];
    run_layer(t, OFF_W1, KIN);
    read_row(reinterpret_cast<const float *>(smem + OFF_B1), z);
#pragma unroll
    for (int i = 0; i < H; i++)
      z[i] = silu(z[i]);
    put_row(t, z);
    run_layer(t, OFF_W2, H);
    read_row(reinterpret_cast<const float *>(smem + OFF_B2), z);
#pragma unroll
    for (int i = 0; i < H; i++)
      z[i] = silu(z[i]);
    put_row(t, z);
    run_layer(t, OFF_W3, H);
    read_row(reinterpret_cast<const float *>(smem + OFF_B3), z);
    // the accumulators are read: the next use of the columns waits for every thread
    fence_before_sync();
    const float *w4 = reinterpret_cast<const float *>(smem + OFF_W4);
    float y = misc[0];
#pragma unroll
    for (int i = 0; i < H; i++)
      y += w4[i] * silu(z[i]);
    return y;
  }
};

// r = gamma / gamma_max from the network's output (linear, or exp of a
// network trained on ln r)
__device__ __forceinline__ float ratio(const Tile &T, float y)
{
  return reinterpret_cast<const float *>(T.smem + OFF_MISC)[11] != 0.0f ? __expf(fminf(y, 1.0f)) : y;
}

// Block set-up: the image into shared memory by one bulk copy, the mbarrier,
// the tensor-memory columns.  Returns false (and flags err) when the copy did
// not land in time.
__device__ __forceinline__ bool tile_setup(Tile &T, unsigned char *smem, const void *image, uint64_t *bar,
                                           uint32_t *tslot, int *err, uint32_t image_bytes = IMAGE_BYTES,
                                           uint32_t act = OFF_ACT)
{
  const int t = threadIdx.x;
  T.smem = smem;
  T.act = act;
  T.bar = bar;
  T.err = err;
  T.phase = 0;
  T.broken = false;
  if (t == 0)
  {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (t < 32)
    tmem_alloc(tslot);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  T.tmem = *tslot;
  if (t == 0)
  {
    mbar_expect_tx(bar, image_bytes);
    bulk_g2s(smem, image, image_bytes, bar);
  }
  return T.wait();
}

__device__ __forceinline__ void tile_release(Tile &T)
{
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (threadIdx.x < 32)
    tmem_free(T.tmem);
}

// ------------------------------------------------------------ host side

// FP32 -> BF16, round to nearest even (NaN kept quiet)
inline uint16_t host_bf16(float f)
{
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7fffffffu) > 0x7f800000u)
    return (uint16_t)((u >> 16) | 0x40u);
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

inline void put_bf16(unsigned char *img, uint32_t off, float v)
{
  const uint16_t b = host_bf16(v);
  memcpy(img + off, &b, 2);
}

// device image of a network (IMAGE_BYTES)
inline void build_image(const dnl_mlp &n, unsigned char *img)
{
  memset(img, 0, IMAGE_BYTES);
  for (int o = 0; o < H; o++)
  {
    for (int i = 0; i < KIN; i++)
      put_bf16(img, OFF_W1 + canon(o, i, H), i < NIN ? n.w1[o][i] : 0.0f);
    for (int i = 0; i < H; i++)
    {
      put_bf16(img, OFF_W2 + canon(o, i, H), n.w2[o][i]);
      put_bf16(img, OFF_W3 + canon(o, i, H), n.w3[o][i]);
    }
  }
  memcpy(img + OFF_B1, n.b1, H * 4);
  memcpy(img + OFF_B2, n.b2, H * 4);
  memcpy(img + OFF_B3, n.b3, H * 4);
  memcpy(img + OFF_W4, n.w4, H * 4);
  float misc[16] = {0};
  misc[0] = n.b4;
  for (int i = 0; i < NIN; i++)
  {
    misc[1 + i] = n.in_mean[i];
    misc[6 + i] = n.in_scale[i];
  }
  misc[11] = n.out_exp;
  misc[12] = n.in_clip;
  memcpy(img + OFF_MISC, misc, sizeof(misc));
}

} // namespace mlp
