// mlp.cu - training and stand-alone inference of the learned Newton initial
// guess (dnl_mlp.cuh): forward, backward and Adam kernels, and their C ABI
// (dnl_mlp_forward, dnl_mlp_gradients, dnl_mlp_train in include/dnlgpu.h).
//
// Training step = one k_mlp_grad launch over the minibatch (one block per tile
// of 128 pairs: the forward on the tensor cores with the pre-activations kept
// in shared memory, the backward through the hidden layers as tensor-core
// products with the transposed weights, the weight gradients as FP32 sums on
// the CUDA cores, one partial gradient per block) and one k_mlp_adam launch
// (fixed-order sum of the partials, Adam on FP32 master weights, BF16 images
// for the next step).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "dnl_kernels.cuh"
#include "dnlgpu.h"

void dnl_internal_set_error(const char *msg);

namespace dnl_train
{
using namespace dnl;
using namespace dnl::mlp;

// parameter vector = the leading floats of dnl_mlp
constexpr int P_W1 = 0, P_B1 = P_W1 + H * KIN, P_W2 = P_B1 + H, P_B2 = P_W2 + H * H, P_W3 = P_B2 + H,
              P_B3 = P_W3 + H * H, P_W4 = P_B3 + H, P_B4 = P_W4 + H, NPARAM = P_B4 + 1;
static_assert(NPARAM * 4 == offsetof(dnl_mlp, in_mean), "parameter vector = leading floats of dnl_mlp");

// training shared memory: image + transposes, A operand tile, pre-activations,
// bf16 copies of the layer inputs for the weight gradients, output gradients
constexpr uint32_t T_ACT = ((IMAGE_BYTES + TRANS_BYTES) + 127) & ~127u;
constexpr int ZP = H + 1; // padded row of the pre-activation arrays
constexpr uint32_t T_Z = T_ACT + ACT_BYTES;    // 3 x M x ZP fp32
constexpr uint32_t T_H = T_Z + 3 * M * ZP * 4; // 2 x M x H bf16 row-major (h1, h2)
constexpr uint32_t T_X = T_H + 2 * M * H * 2;  // M x KIN bf16 row-major (normalised input)
constexpr uint32_t T_DY = T_X + M * KIN * 2;   // M fp32
constexpr uint32_t T_BYTES = T_DY + M * 4;
static_assert(T_BYTES <= 227 * 1024, "training tile fits in shared memory");

// One block = one tile of 128 pairs: forward, backward, weight gradients of the
// tile into part[blockIdx.x][NPARAM] and its squared-error sum into lossp[blockIdx.x].
// idx (may be null) maps tile rows to pairs; rows at or past n count zero.
// scale = 2 / (pairs of the minibatch).
__global__ void __launch_bounds__(TILE, 1) k_mlp_grad(const void *image, const float *x, const float *target,
                                                       const int *idx, long long first, long long n, float scale,
                                                       float *part, float *lossp, int *err)
{
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tslot;
  __shared__ float red[4];
  const int t = threadIdx.x;
  Tile T;
  tile_setup(T, sm, image, &bar, &tslot, err, IMAGE_BYTES + TRANS_BYTES, T_ACT);
  float *Z = reinterpret_cast<float *>(sm + T_Z);
  __nv_bfloat16 *Hb = reinterpret_cast<__nv_bfloat16 *>(sm + T_H);
  __nv_bfloat16 *Xb = reinterpret_cast<__nv_bfloat16 *>(sm + T_X);
  float *DY = reinterpret_cast<float *>(sm + T_DY);
  const float *misc = reinterpret_cast<const float *>(sm + OFF_MISC);
  const float *w4 = reinterpret_cast<const float *>(sm + OFF_W4);

  const long long r = first + (long long)blockIdx.x * M + t;
  const bool live = r < n;
  const long long s = live ? (idx ? (long long)idx[r] : r) : 0;
  float xr[NIN] = {0.f, 0.f, 0.f, 0.f, 0.f};
  float tr = 0.f;
  if (live)
  {
#pragma unroll
    for (int i = 0; i < NIN; i++)
      xr[i] = x[s * NIN + i];
    tr = target[s];
  }
  // ---- forward, keeping the pre-activations and the bf16 layer inputs
  float xin[KIN];
  T.put_input(t, xr, xin);
#pragma unroll
  for (int i = 0; i < KIN; i++)
    Xb[t * KIN + i] = __float2bfloat16_rn(xin[i]);
  float z[H];
#pragma unroll
  for (int l = 0; l < 3; l++)
  {
    const uint32_t wo = l == 0 ? OFF_W1 : (l == 1 ? OFF_W2 : OFF_W3);
    const uint32_t bo = l == 0 ? OFF_B1 : (l == 1 ? OFF_B2 : OFF_B3);
    T.run_layer(t, wo, l == 0 ? KIN : H);
    T.read_row(reinterpret_cast<const float *>(sm + bo), z);
#pragma unroll
    for (int i = 0; i < H; i++)
      Z[(l * M + t) * ZP + i] = z[i];
    if (l < 2)
    {
#pragma unroll
      for (int i = 0; i < H; i++)
      {
        z[i] = silu(z[i]);
        Hb[(l * M + t) * H + i] = __float2bfloat16_rn(z[i]);
      }
      T.put_row(t, z);
    }
  }
  fence_before_sync();
  float y = misc[0];
#pragma unroll
  for (int i = 0; i < H; i++)
    y += w4[i] * silu(z[i]);
  const float dy = live ? scale * (y - tr) : 0.f;
  DY[t] = dy;
  float se = live ? (y - tr) * (y - tr) : 0.f;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    se += __shfl_xor_sync(0xffffffffu, se, o);
  if ((t & 31) == 0)
    red[t >> 5] = se;
  __syncthreads();
  float *pg = part + (size_t)blockIdx.x * NPARAM;
  if (t == 0)
    lossp[blockIdx.x] = red[0] + red[1] + red[2] + red[3];
  // ---- output layer gradients: dw4[j] = sum_b dy_b silu(z3[b][j]), db4 = sum_b dy_b
  if (t < H)
  {
    float acc = 0.f;
    for (int b = 0; b < M; b++)
      acc += DY[b] * silu(Z[(2 * M + b) * ZP + t]);
    pg[P_W4 + t] = acc;
  }
  else if (t == H)
  {
    float acc = 0.f;
    for (int b = 0; b < M; b++)
      acc += DY[b];
    pg[P_B4] = acc;
  }
  __syncthreads();
  // ---- back through the hidden layers: dz3 -> dh2 = dz3 W3 -> dz2 -> dh1 = dz2 W2 -> dz1
#pragma unroll
  for (int i = 0; i < H; i++)
  {
    float *zp = &Z[(2 * M + t) * ZP + i];
    z[i] = dy * w4[i] * silu_grad(*zp);
    *zp = z[i];
  }
  const float zero[H] = {};
#pragma unroll
  for (int l = 1; l >= 0; l--)
  {
    T.put_row(t, z);
    T.run_layer(t, IMAGE_BYTES + (l == 1 ? OFF_W3T : OFF_W2T), H);
    T.read_row(zero, z);
#pragma unroll
    for (int i = 0; i < H; i++)
    {
      float *zp = &Z[(l * M + t) * ZP + i];
      z[i] *= silu_grad(*zp);
      *zp = z[i];
    }
  }
  fence_before_sync();
  __syncthreads();
  // ---- weight gradients of the tile (FP32 sums over its 128 rows)
  {
    const int o = t >> 1, i0 = (t & 1) * (H / 2);
    for (int l = 2; l >= 1; l--) // dW3 = dz3^T h2, dW2 = dz2^T h1
    {
      float acc[H / 2];
#pragma unroll
      for (int k = 0; k < H / 2; k++)
        acc[k] = 0.f;
      float db = 0.f;
      for (int b = 0; b < M; b++)
      {
        const float d = Z[(l * M + b) * ZP + o];
        const __nv_bfloat162 *hr = reinterpret_cast<const __nv_bfloat162 *>(Hb + ((l - 1) * M + b) * H + i0);
#pragma unroll
        for (int k = 0; k < H / 4; k++)
        {
          const float2 hv = __bfloat1622float2(hr[k]);
          acc[2 * k] += d * hv.x;
          acc[2 * k + 1] += d * hv.y;
        }
        db += d;
      }
      const int pw = l == 2 ? P_W3 : P_W2, pb = l == 2 ? P_B3 : P_B2;
#pragma unroll
      for (int k = 0; k < H / 2; k++)
        pg[pw + o * H + i0 + k] = acc[k];
      if ((t & 1) == 0)
        pg[pb + o] = db;
    }
    // dW1 = dz1^T x (inputs 0..15, the padding gets zero), db1
    const int j0 = (t & 1) * (KIN / 2);
    float acc[KIN / 2];
#pragma unroll
    for (int k = 0; k < KIN / 2; k++)
      acc[k] = 0.f;
    float db = 0.f;
    for (int b = 0; b < M; b++)
    {
      const float d = Z[b * ZP + o];
#pragma unroll
      for (int k = 0; k < KIN / 2; k++)
        acc[k] += d * __bfloat162float(Xb[b * KIN + j0 + k]);
      db += d;
    }
#pragma unroll
    for (int k = 0; k < KIN / 2; k++)
      pg[P_W1 + o * KIN + j0 + k] = acc[k];
    if ((t & 1) == 0)
      pg[P_B1 + o] = db;
  }
  tile_release(T);
}

// fixed-order sum of the per-tile partials
__device__ __forceinline__ float sum_parts(const float *part, int nPart, int p)
{
  float g = 0.f;
  for (int c = 0; c < nPart; c++)
    g += part[(size_t)c * NPARAM + p];
  return g;
}

// write parameter p of the master vector into the bf16 / fp32 images
__device__ __forceinline__ void to_image(unsigned char *img, int p, float w)
{
  if (p < P_B1)
  {
    const int o = p / KIN, i = p % KIN;
    *reinterpret_cast<__nv_bfloat16 *>(img + OFF_W1 + canon(o, i, H)) = __float2bfloat16_rn(w);
  }
  else if (p < P_W2)
    reinterpret_cast<float *>(img + OFF_B1)[p - P_B1] = w;
  else if (p < P_B2)
  {
    const int o = (p - P_W2) / H, i = (p - P_W2) % H;
    *reinterpret_cast<__nv_bfloat16 *>(img + OFF_W2 + canon(o, i, H)) = __float2bfloat16_rn(w);
    *reinterpret_cast<__nv_bfloat16 *>(img + IMAGE_BYTES + OFF_W2T + canon(i, o, H)) = __float2bfloat16_rn(w);
  }
  else if (p < P_W3)
    reinterpret_cast<float *>(img + OFF_B2)[p - P_B2] = w;
  else if (p < P_B3)
  {
    const int o = (p - P_W3) / H, i = (p - P_W3) % H;
    *reinterpret_cast<__nv_bfloat16 *>(img + OFF_W3 + canon(o, i, H)) = __float2bfloat16_rn(w);
    *reinterpret_cast<__nv_bfloat16 *>(img + IMAGE_BYTES + OFF_W3T + canon(i, o, H)) = __float2bfloat16_rn(w);
  }
  else if (p < P_W4)
    reinterpret_cast<float *>(img + OFF_B3)[p - P_B3] = w;
  else if (p < P_B4)
    reinterpret_cast<float *>(img + OFF_W4)[p - P_W4] = w;
  else
    reinterpret_cast<float *>(img + OFF_MISC)[0] = w;
}

// gradient vector + squared-error sum of one launch of k_mlp_grad
__global__ void k_mlp_reduce(const float *part, const float *lossp, int nPart, float *grad, float *loss)
{
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < NPARAM)
    grad[p] = sum_parts(part, nPart, p);
  if (p == 0)
  {
    float l = 0.f;
    for (int c = 0; c < nPart; c++)
      l += lossp[c];
    *loss = l;
  }
}

// Adam step `step` (1-based) on the master vector w with moments m, v; images refreshed
__global__ void k_mlp_adam(const float *part, const float *lossp, int nPart, float *w, float *m, float *v,
                           unsigned char *img, float lr, int step, float inv_batch, float *loss_out)
{
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0)
  {
    float l = 0.f;
    for (int c = 0; c < nPart; c++)
      l += lossp[c];
    *loss_out = l * inv_batch;
  }
  if (p >= NPARAM)
    return;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float g = sum_parts(part, nPart, p);
  const float mm = b1 * m[p] + (1.f - b1) * g;
  const float vv = b2 * v[p] + (1.f - b2) * g * g;
  m[p] = mm;
  v[p] = vv;
  const float mh = mm / (1.f - powf(b1, (float)step));
  const float vh = vv / (1.f - powf(b2, (float)step));
  float wn = w[p] - lr * mh / (sqrtf(vh) + eps);
  if (p < P_B1 && (p % KIN) >= NIN)
    wn = 0.f; // padding columns of the first layer stay zero
  w[p] = wn;
  to_image(img, p, wn);
}

// stand-alone inference: persistent over tiles of 128 inputs
__global__ void __launch_bounds__(TILE) k_mlp_forward(const void *image, const float *x, long long n, float *y,
                                                      int *err)
{
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tslot;
  const int t = threadIdx.x;
  Tile T;
  tile_setup(T, sm, image, &bar, &tslot, err);
  const long long tiles = (n + M - 1) / M;
  for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x)
  {
    const long long r = tile * M + t;
    float xr[NIN] = {0.f, 0.f, 0.f, 0.f, 0.f};
    if (r < n)
#pragma unroll
      for (int i = 0; i < NIN; i++)
        xr[i] = x[r * NIN + i];
    const float out = T.forward(t, xr);
    if (r < n)
      y[r] = out;
  }
  tile_release(T);
}

// ------------------------------------------------------------------ host

struct Work
{
  std::vector<void *> allocs;
  ~Work()
  {
    for (void *p : allocs)
      cudaFree(p);
  }
  template <typename T> bool alloc(T **p, size_t n)
  {
    if (cudaMalloc((void **)p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess)
      return false;
    allocs.push_back(*p);
    return true;
  }
};

int fail_msg(int code, const char *msg)
{
  dnl_internal_set_error(msg);
  return code;
}

#define MCK(call)                                                                                                 \
  do                                                                                                              \
  {                                                                                                               \
    cudaError_t e_ = (call);                                                                                      \
    if (e_ != cudaSuccess)                                                                                        \
    {                                                                                                             \
      char b_[256];                                                                                               \
      snprintf(b_, sizeof(b_), "%s failed: %s", #call, cudaGetErrorString(e_));                                   \
      return fail_msg(DNL_ERR_CUDA, b_);                                                                          \
    }                                                                                                             \
  } while (0)

void host_train_image(const dnl_mlp &net, std::vector<unsigned char> &img)
{
  img.assign(IMAGE_BYTES + TRANS_BYTES, 0);
  build_image(net, img.data());
  for (int o = 0; o < H; o++)
    for (int i = 0; i < H; i++)
    {
      put_bf16(img.data(), IMAGE_BYTES + OFF_W2T + canon(i, o, H), net.w2[o][i]);
      put_bf16(img.data(), IMAGE_BYTES + OFF_W3T + canon(i, o, H), net.w3[o][i]);
    }
}

int check_err_flag(int *derr, cudaStream_t st)
{
  int e = 0;
  MCK(cudaMemcpyAsync(&e, derr, sizeof(int), cudaMemcpyDeviceToHost, st));
  MCK(cudaStreamSynchronize(st));
  if (e)
    return fail_msg(DNL_ERR_CUDA, "a tensor-core or bulk-copy wait of the network kernels did not complete in time");
  return DNL_OK;
}

bool set_grad_smem()
{
  static bool done = false;
  if (!done)
    done = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T_BYTES) == cudaSuccess;
  return done;
}

} // namespace dnl_train

using namespace dnl_train;

extern "C" {

int dnl_mlp_forward(const dnl_mlp *net, const float *d_x, int64_t n, float *d_y, void *stream)
{
  if (!net || n < 0 || (n > 0 && (!d_x || !d_y)))
    return fail_msg(DNL_ERR_ARG, "dnl_mlp_forward: invalid argument");
  if (n == 0)
    return DNL_OK;
  cudaStream_t st = (cudaStream_t)stream;
  Work w;
  unsigned char *dimg;
  int *derr;
  if (!w.alloc(&dimg, IMAGE_BYTES) || !w.alloc(&derr, 1))
    return fail_msg(DNL_ERR_CUDA, "dnl_mlp_forward: cudaMalloc failed");
  std::vector<unsigned char> img(IMAGE_BYTES);
  build_image(*net, img.data());
  MCK(cudaMemcpyAsync(dimg, img.data(), IMAGE_BYTES, cudaMemcpyHostToDevice, st));
  MCK(cudaMemsetAsync(derr, 0, sizeof(int), st));
  MCK(cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES));
  int perSM = 0, dev = 0, sms = 0;
  MCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_mlp_forward, TILE, SMEM_BYTES));
  MCK(cudaGetDevice(&dev));
  MCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  // the blocks resident on one SM must find their tensor-memory columns free
  if (perSM * (int)TMEM_COLS > 512)
    return fail_msg(DNL_ERR_CUDA, "dnl_mlp_forward: too many blocks per SM for the tensor memory");
  perSM = std::max(1, perSM);
  const long long tiles = (n + TILE - 1) / TILE;
  const int grid = (int)std::min<long long>(tiles, (long long)perSM * sms);
  k_mlp_forward<<<grid, TILE, SMEM_BYTES, st>>>(dimg, d_x, n, d_y, derr);
  MCK(cudaGetLastError());
  return check_err_flag(derr, st);
}

int dnl_mlp_gradients(const dnl_mlp *net, const float *d_x, const float *d_t, int64_t n, dnl_mlp *grad, float *loss,
                      void *stream)
{
  if (!net || !grad || n <= 0 || !d_x || !d_t)
    return fail_msg(DNL_ERR_ARG, "dnl_mlp_gradients: invalid argument");
  cudaStream_t st = (cudaStream_t)stream;
  const long long tiles = (n + TILE - 1) / TILE;
  if (tiles > (1 << 20))
    return fail_msg(DNL_ERR_ARG, "dnl_mlp_gradients: too many samples for one call");
  Work w;
  unsigned char *dimg;
  float *part, *lossp, *dgrad, *dloss;
  int *derr;
  if (!w.alloc(&dimg, IMAGE_BYTES + TRANS_BYTES) || !w.alloc(&part, (size_t)tiles * NPARAM) ||
      !w.alloc(&lossp, tiles) || !w.alloc(&dgrad, NPARAM) || !w.alloc(&dloss, 1) || !w.alloc(&derr, 1))
    return fail_msg(DNL_ERR_CUDA, "dnl_mlp_gradients: cudaMalloc failed");
  std::vector<unsigned char> img;
  host_train_image(*net, img);
  MCK(cudaMemcpyAsync(dimg, img.data(), img.size(), cudaMemcpyHostToDevice, st));
  MCK(cudaMemsetAsync(derr, 0, sizeof(int), st));
  if (!set_grad_smem())
    return fail_msg(DNL_ERR_CUDA, "dnl_mlp_gradients: shared memory attribute refused");
  k_mlp_grad<<<(int)tiles, TILE, T_BYTES, st>>>(dimg, d_x, d_t, nullptr, 0, n, 2.0f / (float)n, part, lossp, derr);
  MCK(cudaGetLastError());
  k_mlp_reduce<<<(NPARAM + 255) / 256, 256, 0, st>>>(part, lossp, (int)tiles, dgrad, dloss);
  MCK(cudaGetLastError());
  int rc = check_err_flag(derr, st);
  if (rc)
    return rc;
  memset(grad, 0, sizeof(dnl_mlp));
  MCK(cudaMemcpyAsync(grad, dgrad, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, st));
  float l = 0.f;
  MCK(cudaMemcpyAsync(&l, dloss, sizeof(float), cudaMemcpyDeviceToHost, st));
  MCK(cudaStreamSynchronize(st));
  if (loss)
    *loss = l / (float)n;
  return DNL_OK;
}

int dnl_mlp_train(dnl_mlp *net, const float *d_x, const float *d_t, int64_t n, int32_t epochs, int32_t batch_tiles,
                  float learning_rate, uint64_t seed, float *loss_history, void *stream)
{
  if (!net || !d_x || !d_t || n <= 0 || epochs < 0 || batch_tiles < 1 || batch_tiles > 4096 || n > (1ll << 31) - 1)
    return fail_msg(DNL_ERR_ARG, "dnl_mlp_train: invalid argument");
  cudaStream_t st = (cudaStream_t)stream;
  const long long batch = (long long)batch_tiles * TILE;
  const long long steps = (n + batch - 1) / batch;
  Work w;
  unsigned char *dimg;
  float *part, *lossp, *dw, *dm, *dv, *dstep_loss;
  int *derr, *dperm;
  if (!w.alloc(&dimg, IMAGE_BYTES + TRANS_BYTES) || !w.alloc(&part, (size_t)batch_tiles * NPARAM) ||
      !w.alloc(&lossp, batch_tiles) || !w.alloc(&dw, NPARAM) || !w.alloc(&dm, NPARAM) || !w.alloc(&dv, NPARAM) ||
      !w.alloc(&dstep_loss, (size_t)std::max<long long>(steps * epochs, 1)) || !w.alloc(&derr, 1) ||
      !w.alloc(&dperm, n))
    return fail_msg(DNL_ERR_CUDA, "dnl_mlp_train: cudaMalloc failed");
  std::vector<unsigned char> img;
  host_train_image(*net, img);
  MCK(cudaMemcpyAsync(dimg, img.data(), img.size(), cudaMemcpyHostToDevice, st));
  MCK(cudaMemcpyAsync(dw, net, NPARAM * sizeof(float), cudaMemcpyHostToDevice, st));
  MCK(cudaMemsetAsync(dm, 0, NPARAM * sizeof(float), st));
  MCK(cudaMemsetAsync(dv, 0, NPARAM * sizeof(float), st));
  MCK(cudaMemsetAsync(derr, 0, sizeof(int), st));
  if (!set_grad_smem())
    return fail_msg(DNL_ERR_CUDA, "dnl_mlp_train: shared memory attribute refused");
  std::vector<int> perm((size_t)n);
  std::mt19937_64 rng(seed);
  int step = 0;
  for (int ep = 0; ep < epochs; ep++)
  {
    for (long long i = 0; i < n; i++)
      perm[(size_t)i] = (int)i;
    std::shuffle(perm.begin(), perm.end(), rng);
    MCK(cudaMemcpyAsync(dperm, perm.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, st));
    for (long long b = 0; b < steps; b++)
    {
      const long long first = b * batch;
      const long long rows = std::min(batch, n - first);
      const int tiles = (int)((rows + TILE - 1) / TILE);
      k_mlp_grad<<<tiles, TILE, T_BYTES, st>>>(dimg, d_x, d_t, dperm, first, n, 2.0f / (float)rows, part, lossp,
                                               derr);
      step++;
      k_mlp_adam<<<(NPARAM + 255) / 256, 256, 0, st>>>(part, lossp, tiles, dw, dm, dv, dimg, learning_rate, step,
                                                       1.0f / (float)rows, dstep_loss + (step - 1));
    }
    MCK(cudaGetLastError());
    // the permutation buffer is refilled for the next epoch: wait for this one
    MCK(cudaStreamSynchronize(st));
  }
  int rc = check_err_flag(derr, st);
  if (rc)
    return rc;
  MCK(cudaMemcpyAsync(net, dw, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, st));
  std::vector<float> sl((size_t)std::max<long long>(steps * epochs, 1));
  MCK(cudaMemcpyAsync(sl.data(), dstep_loss, sl.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
  MCK(cudaStreamSynchronize(st));
  if (loss_history)
    for (int ep = 0; ep < epochs; ep++)
    {
      double s = 0.0;
      for (long long b = 0; b < steps; b++)
        s += sl[(size_t)(ep * steps + b)];
      loss_history[ep] = (float)(s / (double)steps);
    }
  return DNL_OK;
}

} // extern "C"
