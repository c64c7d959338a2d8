// static_pass.cu - element pass on caller-owned device arrays that allocates
// no device memory (dnl_element_pass_static, include/dnlgpu.h).
//
// Some callers cannot allocate device memory: a host code that hands the GPU
// to a memory manager of its own and forbids any other allocation, or one that
// calls between stream captures where a cudaMalloc would synchronize the
// device.  They pass their inputs and outputs as device pointers; the scratch
// this pass needs (the per element-node force slots, the node -> slot lists
// built from the connectivity and a small control block) lives in the
// file-scope array below, sized for at most DNL_STATIC_MAX_ELEMS elements and
// DNL_STATIC_MAX_NODES nodes.  Every GPU that loads the library holds it until
// the process exits.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "dnl_kernels.cuh"
#include "dnlgpu.h"

using namespace dnl;

void dnl_internal_set_error(const char *msg); // engine.cu

namespace dnl_static
{
constexpr int MAX_ELEMS = DNL_STATIC_MAX_ELEMS;
constexpr int MAX_NODES = DNL_STATIC_MAX_NODES;
constexpr int MAX_IPS = MAX_ELEMS * 8;

// layout of the scratch array (byte offsets)
constexpr size_t OFF_CTL = 0;
constexpr size_t OFF_SLOT = 256;
constexpr size_t OFF_COUNT = OFF_SLOT + sizeof(double4) * MAX_IPS;
constexpr size_t OFF_CURSOR = OFF_COUNT + sizeof(int) * (MAX_NODES + 1);
constexpr size_t OFF_LIST = OFF_CURSOR + sizeof(int) * MAX_NODES;
constexpr size_t OFF_MAT = (OFF_LIST + sizeof(int) * MAX_IPS + 255) / 256 * 256;
constexpr size_t SCRATCH_BYTES = OFF_MAT + sizeof(MatDev);

// The scratch of every call (about 5.3 MB).  Host code only takes its device
// address (cudaGetSymbolAddress); the kernels receive that address.
static __device__ __align__(256) unsigned char g_scratch[SCRATCH_BYTES];

struct Scratch
{
  Ctl *ctl;
  double4 *slot;
  int *count, *cursor, *list;
  MatDev *mat; // the call's material, read by the return from global memory
};

__host__ __device__ Scratch carve(unsigned char *base)
{
  return Scratch{reinterpret_cast<Ctl *>(base + OFF_CTL), reinterpret_cast<double4 *>(base + OFF_SLOT),
                 reinterpret_cast<int *>(base + OFF_COUNT), reinterpret_cast<int *>(base + OFF_CURSOR),
                 reinterpret_cast<int *>(base + OFF_LIST), reinterpret_cast<MatDev *>(base + OFF_MAT)};
}

// Caller's arrays: point state component-major [29][n_ips] FP64, nodes [n][3].
struct StaticIo
{
  const double *coords, *du;
  double *ip;
  double4 *slots;
  const MatDev *mat_;
  int nIP, q;
  __device__ __forceinline__ double4 x(int n) const
  {
    return make_double4(coords[3 * n], coords[3 * n + 1], coords[3 * n + 2], 0.0);
  }
  __device__ __forceinline__ double4 u(int n) const
  {
    return make_double4(du[3 * n], du[3 * n + 1], du[3 * n + 2], 0.0);
  }
  __device__ __forceinline__ const MatDev &mat(int) const { return *mat_; }
  __device__ __forceinline__ const MatDev *matp(int) const { return mat_; }
  __device__ __forceinline__ JC<double> law(int) const
  {
    JC<double> j;
    j.load(*mat_);
    return j;
  }
  __device__ __forceinline__ double rho0(int) const { return mat_->rho0; }
  __device__ __forceinline__ void put(int c, double v) const { ip[(size_t)c * nIP + q] = v; }
  __device__ __forceinline__ void slot(const double4 &v) const { slots[q] = v; }
  __device__ __forceinline__ const float *ip32() const { return nullptr; }
  __device__ __forceinline__ void first_node(unsigned amask, int base, const double4 &X, const double4 &U,
                                             double4 &X0, double4 &U0) const
  {
    first_node_by_shuffle(amask, base, X, U, X0, U0);
  }
};

struct PlainState
{
  const double *ip;
  int nIP, q;
  __device__ __forceinline__ double operator()(int c) const { return ip[(size_t)c * nIP + q]; }
};

struct Args
{
  const double *coords, *du;
  const int *conn;
  double *ip, *force;
  int nN, nE, npe;
  double dt;
  MatDev mat;
  unsigned char *scratch;
};

// control block, node slot counts set to zero (the array keeps the last call's contents)
__global__ void k_sp_clear(Args a)
{
  Scratch s = carve(a.scratch);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0)
  {
    Ctl c;
    memset(&c, 0, sizeof(c));
    c.active = 1;
    c.dt_eff = a.dt;
    *s.ctl = c;
    *s.mat = a.mat;
  }
  if (i <= a.nN)
    s.count[i] = 0;
}

// Node slot counts.  The connectivity is the caller's device array: an entry
// outside [0, n_nodes) is not counted, and the call reports DNL_ERR_ARG with
// the element in the control block; the kernels after this one then leave at
// once, so no index taken from the connectivity reaches memory unchecked.
__global__ void k_sp_count(Args a)
{
  Scratch s = carve(a.scratch);
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= a.nE * a.npe)
    return;
  const int n = a.conn[k];
  if ((unsigned)n < (unsigned)a.nN)
    atomicAdd(&s.count[n + 1], 1);
  else
    raise_status(s.ctl, DNL_ERR_ARG, k / a.npe);
}

// true once k_sp_count has found a connectivity entry out of range.  Only
// k_sp_count sets DNL_ERR_ARG, and it completes before the kernels that test
// it start, so every thread of a launch reads the same answer (the element
// kernel may raise other codes while it runs; those do not stop the pass).
__device__ __forceinline__ bool bad_input(const Scratch &s)
{
  return *(volatile int *)&s.ctl->status == DNL_ERR_ARG;
}

// exclusive offsets of the node slot lists (one block)
__global__ void k_sp_scan(Args a)
{
  Scratch s = carve(a.scratch);
  if (bad_input(s))
    return;
  __shared__ int part[1024];
  const int n = a.nN + 1, t = threadIdx.x, per = (n + blockDim.x - 1) / blockDim.x;
  const int b = t * per, e = min(n, b + per);
  int acc = 0;
  for (int i = b; i < e; i++)
    acc += s.count[i];
  part[t] = acc;
  __syncthreads();
  if (t == 0)
  {
    int run = 0;
    for (int k = 0; k < (int)blockDim.x; k++)
    {
      const int v = part[k];
      part[k] = run;
      run += v;
    }
  }
  __syncthreads();
  int run = part[t];
  for (int i = b; i < e; i++)
  {
    run += s.count[i];
    s.count[i] = run; // count[i] now holds the end of node i-1's list = start of node i's
  }
  __syncthreads();
  for (int i = t; i < a.nN; i += blockDim.x)
    s.cursor[i] = s.count[i];
}

__global__ void k_sp_fill(Args a)
{
  Scratch s = carve(a.scratch);
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < a.nE * a.npe && !bad_input(s))
    s.list[atomicAdd(&s.cursor[a.conn[k]], 1)] = k;
}

// each node's slots in increasing element order (the reference's assembly order)
__global__ void k_sp_sort(Args a)
{
  Scratch s = carve(a.scratch);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nN || bad_input(s))
    return;
  int *L = s.list + s.count[i];
  const int n = s.count[i + 1] - s.count[i];
  for (int j = 1; j < n; j++)
  {
    const int v = L[j];
    int k = j - 1;
    while (k >= 0 && L[k] > v)
    {
      L[k + 1] = L[k];
      k--;
    }
    L[k + 1] = v;
  }
}

template <int NPE> __global__ void __launch_bounds__(TILE) k_sp_element(Args a)
{
  constexpr int ROW = ElemShape<NPE>::template pass_row<double>;
  __shared__ double sh[TILE * ROW];
  Scratch s = carve(a.scratch);
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const int g = lane & (NPE - 1);
  const int base = lane & ~(NPE - 1);
  const int e = q / NPE;
  const bool act = e < a.nE && !bad_input(s);
  const unsigned amask = __ballot_sync(0xffffffffu, act);
  if (!act)
    return;
  const int nIP = a.nE * NPE;
  StaticIo io{a.coords, a.du, a.ip, s.slot, s.mat, nIP, q};
  PlainState old{a.ip, nIP, q};
  element_update<double, NPE>(io, s.ctl, q, e, g, base, amask, a.conn[q], old, sh + threadIdx.x * ROW,
                              sh + (threadIdx.x - g) * ROW);
}

__global__ void k_sp_gather(Args a)
{
  Scratch s = carve(a.scratch);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nN || bad_input(s))
    return;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  for (int k = s.count[i]; k < s.count[i + 1]; k++)
  {
    const double4 v = s.slot[s.list[k]];
    fx += v.x;
    fy += v.y;
    fz += v.z;
  }
  a.force[3 * i] = fx;
  a.force[3 * i + 1] = fy;
  a.force[3 * i + 2] = fz;
}

std::mutex g_setup_mutex;
unsigned char *g_scratch_addr[128] = {nullptr};

// Device address of the scratch on the current device, looked up once per
// device (the first call on a device does it, so make that call before any
// stream capture).
int scratch_address(unsigned char **out)
{
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128)
  {
    cudaGetLastError();
    dnl_internal_set_error("dnl_element_pass_static: no current CUDA device");
    return DNL_ERR_NO_DEVICE;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev])
  {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p)
    {
      char buf[256];
      snprintf(buf, sizeof(buf), "dnl_element_pass_static: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
      dnl_internal_set_error(buf);
      return DNL_ERR_CUDA;
    }
    g_scratch_addr[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_scratch_addr[dev];
  return DNL_OK;
}
} // namespace dnl_static

using namespace dnl_static;

extern "C" int dnl_element_pass_static(int32_t elem_type, int32_t n_nodes, int32_t n_elems, const double *d_coords,
                                       const double *d_du, const int32_t *d_conn, const dnl_material *material,
                                       double time_step, double *d_ips, double *d_force, void *stream)
{
  const int npe = elem_type == DNL_ELHEX8N3D ? 8 : (elem_type == DNL_ELQUA4NAX ? 4 : 0);
  char buf[256];
  if (npe == 0 || n_nodes <= 0 || n_elems <= 0 || !d_coords || !d_du || !d_conn || !material || !d_ips ||
      !d_force || !(time_step > 0.0))
  {
    dnl_internal_set_error("dnl_element_pass_static: invalid argument");
    return DNL_ERR_ARG;
  }
  if (n_elems > MAX_ELEMS || n_nodes > MAX_NODES)
  {
    snprintf(buf, sizeof(buf),
             "dnl_element_pass_static: %d elements / %d nodes exceed the static scratch limit of %d elements / "
             "%d nodes",
             n_elems, n_nodes, MAX_ELEMS, MAX_NODES);
    dnl_internal_set_error(buf);
    return DNL_ERR_ARG;
  }
  unsigned char *scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc)
    return rc;
  const dnl_material &m = *material;
  Args a;
  a.coords = d_coords;
  a.du = d_du;
  a.conn = d_conn;
  a.ip = d_ips;
  a.force = d_force;
  a.nN = n_nodes;
  a.nE = n_elems;
  a.npe = npe;
  a.dt = time_step;
  a.scratch = scratch;
  a.mat = make_mat(m);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nIP = n_elems * npe;
  k_sp_clear<<<(n_nodes + 1 + 255) / 256, 256, 0, st>>>(a);
  k_sp_count<<<(nIP + 255) / 256, 256, 0, st>>>(a);
  k_sp_scan<<<1, 1024, 0, st>>>(a);
  k_sp_fill<<<(nIP + 255) / 256, 256, 0, st>>>(a);
  k_sp_sort<<<(n_nodes + 255) / 256, 256, 0, st>>>(a);
  if (npe == 8)
    k_sp_element<8><<<(nIP + TILE - 1) / TILE, TILE, 0, st>>>(a);
  else
    k_sp_element<4><<<(nIP + TILE - 1) / TILE, TILE, 0, st>>>(a);
  k_sp_gather<<<(n_nodes + 255) / 256, 256, 0, st>>>(a);
  cudaError_t e = cudaGetLastError();
  int status = 0;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&status, &carve(scratch).ctl->status, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(st);
  if (e != cudaSuccess)
  {
    snprintf(buf, sizeof(buf), "dnl_element_pass_static: %s", cudaGetErrorString(e));
    dnl_internal_set_error(buf);
    return DNL_ERR_CUDA;
  }
  if (status != 0)
  {
    dnl_internal_set_error(status == DNL_ERR_ARG ? "dnl_element_pass_static: connectivity entry outside [0, n_nodes)"
                           : status == DNL_ERR_NEG_JACOBIAN ? "dnl_element_pass_static: negative Jacobian"
                                                            : "dnl_element_pass_static: radial return failed");
    return status;
  }
  return DNL_OK;
}
