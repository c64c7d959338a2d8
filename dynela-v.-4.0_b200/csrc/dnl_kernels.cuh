// dnl_kernels.cuh - sm_100a kernels of one explicit increment.
//
// Per increment (one CUDA-graph replay):
//   [k_bc_prep]   imposed-speed nodes: field0 values of the predictor BC
//   k_element     strains, pressure, radial return, rotation, density, element forces
//   k_nodal       CSR gather of element forces, Chung-Hulbert predictor+corrector, BCs
//   k_courant     critical time step (only when due), warp-shuffle min + atomicMin
//   k_control     end of step / start of the next one (time, dt, increment, swap)
//
// Data layout in HBM (all instances concatenated):
//   nodes        double4 AoS (x, y, z, pad): coords, disp, u[2], v[2], a[2]; double mass
//   elements     int32 conn[nE*npe]; int32 material
//   points       Real ip[29][nIPpad] component-major (coalesced per component)
//   force slots  Real4 slot[nE*npe]: one per (element, local node), stored in node
//                order (the slots of a node are contiguous, its elements in
//                increasing order); the element pass scatters to slot_pos[q], the
//                nodal pass reads its node's run of slots
#pragma once

#include <cooperative_groups.h>
#include <cuda_bf16.h>

#include <cstring>

#include "dnl_math.cuh"
#include "dnlgpu.h"

namespace dnl
{
// internal linkage: every translation unit that includes this header gets its
// own copy of the kernels and helpers
namespace
{

// Per-instance solver state, resident on the device.
struct __align__(128) Ctl
{
  double t, dt, t_end, t_stop;  // Model::currentTime, Solver::timeStep, end of solve, pause time
  double dt_eff, t_new;         // time step and end time of the prepared increment
  unsigned long long min_bits;  // atomicMin accumulator of l/c (positive double bits)
  long long inc, inc_stop;      // Solver::currentIncrement, stop increment
  int active, prepared, due, f0; // prepared increment runs / begin evaluated / dt recompute / field0 buffer
  int status, bad, resolves, ts_freq;
  double safety, omegaS, alphaM, beta, gammaN;
  int elem_begin, elem_end, node_begin, node_end;
  int ts_method, pi_iters, direct, plane; // direct: one-step return (Element::computeStressDirect);
                                          // plane: plane-strain quads (no axisymmetric terms)
  double pi_fmax, pi_omega; // power iteration: Model::_powerIterationFreqMax, last omega_max
  double dt_last;           // time step of the last completed increment
};

static constexpr unsigned long long INF_BITS = 0x7ff0000000000000ull;

// Programmatic dependent launch: the kernels of an increment are launched so
// that the next one is scheduled as the blocks of the one before leave; each
// waits here, before its first memory access, until the previous grid has
// completed and its writes are visible (a no-op after a normal launch).  No
// kernel triggers its dependents early: blocks of the next kernel holding
// registers while the previous one still runs slowed the increment.
__device__ __forceinline__ void pdl_wait()
{
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

template <typename R> struct V4;
template <> struct V4<double> { using type = double4; };
template <> struct V4<float> { using type = float4; };

struct DevModel
{
  int nInst, nN, nE, nIP, nIPpad, nSpeed, nFunc;
  int slotW; // force slots per node in the fixed-stride layout (node i's at i * slotW), 0: CSR layout
  const int *inst_elem_begin; // [nInst+1]
  const int *inst_node_begin; // [nInst+1]
  Ctl *ctl;
  double4 *x, *disp;
  double4 *u[2], *v[2], *a[2];
  double *mass;
  const int *conn;
  const int *emat;
  const MatDev *mat;
  void *ip;
  void *slot;
  const int *csr_off;      // [nN+1] prefix sums of the nodes' slot counts (their first slots in the CSR layout)
  const int *slot_pos;     // [nE*npe] slot of (element, local node) in node order
  const uint8_t *bc;       // per node: 2 bits per component (DNL_BC_*)
  const double4 *bcval;    // per node imposed speed (only read where the code is DNL_BC_SPEED)
  const int4 *bcfun;       // per node function index per component (-1 none)
  const int *speed_nodes;  // nodes carrying an imposed speed
  const double *fx, *fy;   // packed function points
  const int *foff;         // [nFunc+1]
  double4 *fout;           // assembled forces (kernel-level entry point)
  // power-iteration time step (single-model engines)
  double *pv, *pv2;        // [nN*3] iteration vectors (dof = 3 node + component)
  double4 *pislot;         // [nE*npe] element K v contributions, node order
  double *blockmax;        // [gridDim] per-block max |v|
  // element-pass modes (learned initial guess, Newton statistics, training pairs)
  const void *mlp_image;   // network image (dnl_mlp.cuh)
  unsigned long long *stats; // [0] yield-function evaluations and [1] yielding points, [2] and [3] the same
                             // over the points of the guess scope
  float *harvest;          // pairs of DNL_MLP_PAIR_WORDS floats
  unsigned long long *harvest_count;
  long long harvest_cap;
  int harvest_stride;
  int guess_scope;         // DNL_GUESS_ALL or DNL_GUESS_FIRST_YIELD
  unsigned *done_count;    // blocks of the fused Courant + end-of-increment kernel that have finished
  unsigned *step_due;      // set by the nodal pass: the Courant pass of this increment has work
  // batches: the instances that run this increment, in index order, and the
  // prefix sums of their point tiles, nodes and elements (k_active_list)
  int *act_count;          // [1]
  int *act_list;           // [nInst]
  int *act_tile_pre, *act_node_pre, *act_elem_pre; // [nInst + 1]
  int *due_count, *due_list, *due_elem_pre;         // the same for the running instances whose time step is due
  // a model with one material: its Johnson-Cook block and density, read by the
  // element pass from the kernel parameters (JC<R, true>)
  JCParams<float> one32;
  JCParams<double> one64;
  double one_rho0;
};

template <typename R> __device__ __forceinline__ const JCParams<R> *one_params(const DevModel &M)
{
  if constexpr (sizeof(R) == 4)
    return &M.one32;
  else
    return &M.one64;
}

// Node i's first force slot: a fixed stride of slotW slots per node when every
// node has at most that many (the padding slots hold zeros, which leave the
// sums unchanged), else the CSR offsets.  The slots of node i are
// [slot_begin(i), slot_begin(i) + csr_off[i+1] - csr_off[i]).
__device__ __forceinline__ int slot_begin(const DevModel &M, int i)
{
  return M.slotW ? M.slotW * i : M.csr_off[i];
}

__device__ __forceinline__ int find_segment(const int *begin, int n, int v)
{
  int lo = 0, hi = n - 1;
  while (lo < hi)
  {
    int mid = (lo + hi + 1) >> 1;
    if (__ldg(begin + mid) <= v)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ double func_value(const DevModel &M, int f, double t)
{
  int b = M.foff[f], e = M.foff[f + 1];
  const double *X = M.fx, *Y = M.fy;
  if (t <= X[b])
    return Y[b];
  for (int i = b + 1; i < e; i++)
    if (X[i] >= t)
    {
      if (X[i] == t)
        return Y[i];
      return ((t - X[i - 1]) / (X[i] - X[i - 1])) * (Y[i] - Y[i - 1]) + Y[i - 1];
    }
  return Y[e - 1];
}

__host__ __device__ __forceinline__ double &comp(double4 &v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }

// --------------------------------------------------------------- helpers

// Sum v[] over the NPE lanes of an element group and leave in lane g the DIM
// values of node g (a butterfly reduce-scatter: NPE/2, NPE/4, ... lanes apart).
template <typename R, int NPE, int DIM>
__device__ __forceinline__ void reduce_scatter(unsigned mask, int g, R (&w)[NPE * DIM])
{
#pragma unroll
  for (int half = NPE / 2; half >= 1; half >>= 1)
  {
    const bool upper = (g & half) != 0;
#pragma unroll
    for (int k = 0; k < half * DIM; k++)
    {
      R send = upper ? w[k] : w[k + half * DIM];
      R keep = upper ? w[k + half * DIM] : w[k];
      w[k] = keep + __shfl_xor_sync(mask, send, half);
    }
  }
}

template <int NPE> __device__ __forceinline__ float group_sum(unsigned mask, float v)
{
#pragma unroll
  for (int h = 1; h < NPE; h <<= 1)
    v += __shfl_xor_sync(mask, v, h);
  return v;
}
template <int NPE> __device__ __forceinline__ double group_sum(unsigned mask, double v)
{
#pragma unroll
  for (int h = 1; h < NPE; h <<= 1)
    v += __shfl_xor_sync(mask, v, h);
  return v;
}

// local coordinate sign of node / Gauss point n along axis k (ElHex8N3D.C:33-90,
// ElQua4NAx.C:28-60): (-,-,-) (+,-,-) (+,+,-) (-,+,-) (-,-,+) (+,-,+) (+,+,+) (-,+,+)
__host__ __device__ constexpr int node_sign(int n, int k)
{
  return k == 0 ? ((n & 3) == 1 || (n & 3) == 2 ? 1 : -1) : (k == 1 ? ((n & 3) >= 2 ? 1 : -1) : (n >= 4 ? 1 : -1));
}

// Point state in tiles of TILE consecutive integration points: within a tile,
// component-major (one TILE-long run per component), so that a tile is one
// contiguous block for a bulk copy and every component access is coalesced.
// Inside a tile the components that the element pass reads come first: the
// pressure and the density (which it only writes) are moved to the last two
// runs, so that the staged passes copy DNL_IP_NREAD of the DNL_IP_NCOMP runs.
// ip_slot maps a component (DNL_IP_*) to its run; the public layout of
// dnl_engine_get_ips / set_ips is unchanged.
constexpr int TILE = 128;
constexpr int DNL_IP_NREAD = DNL_IP_NCOMP - 2;
__host__ __device__ constexpr int ip_slot(int c)
{
  return c < DNL_IP_PRESSURE ? c
         : c == DNL_IP_PRESSURE ? DNL_IP_NCOMP - 2
         : c == DNL_IP_DENSITY  ? DNL_IP_NCOMP - 1
         : c < DNL_IP_DENSITY   ? c - 1
                                : c - 2; // DNL_IP_EINT, DNL_IP_EINEL -> 24, 25; DNL_IP_DETJ0 -> 26
}
static_assert(ip_slot(DNL_IP_EINT) == 24 && ip_slot(DNL_IP_EINEL) == 25 && ip_slot(DNL_IP_DETJ0) == 26 &&
                  ip_slot(DNL_IP_PRESSURE) == 27 && ip_slot(DNL_IP_DENSITY) == 28 && DNL_IP_NCOMP == 29,
              "run order of the point state");
__host__ __device__ __forceinline__ size_t ip_index(int c, int q)
{
  return (size_t)(q / TILE) * (DNL_IP_NCOMP * TILE) + (size_t)ip_slot(c) * TILE + (q % TILE);
}

// The point state streams through the L2 once per increment (143 MB on the
// mixed path, 285 MB in FP64, more than the 126 MB L2): its loads and stores
// are marked evict-first (ld/st.global.cs), so that the force slots, node
// vectors and connectivity that the next passes read stay in the L2.
template <typename R> __device__ __forceinline__ R ipv(const DevModel &M, int c, int q)
{
  return __ldcs(reinterpret_cast<const R *>(M.ip) + ip_index(c, q));
}
template <typename R> __device__ __forceinline__ void ipw(const DevModel &M, int c, int q, R v)
{
  __stcs(reinterpret_cast<R *>(M.ip) + ip_index(c, q), v);
}

__device__ __forceinline__ void raise_status(Ctl *c, int code, int index)
{
  if (atomicCAS(&c->status, 0, code) == 0)
    c->bad = index;
}

// FP64 re-solve of a point whose FP32 return failed its tests.  The point
// state is re-read from global memory (it is written back only after the
// return) and the result comes back by value, so the common path keeps its
// state in registers.
struct Resolved
{
  float s[6];
  float epsp, depsp, gamma, gcum, yield, T, eint, einel, kplast;
  int ok;
};

__device__ __noinline__ Resolved resolve_fp64(const float *ip, int q, const MatDev *matp, float e0, float e1,
                                              float e2, float e3, float e4, float e5, double dt, float pressure)
{
  const MatDev &mp = *matp;
  JC<double> jc;
  jc.load(mp);
  ReturnState<double> d;
  for (int c = 0; c < 6; c++)
    d.s[c] = ip[ip_index(DNL_IP_STRESS + c, q)];
  d.epsp = ip[ip_index(DNL_IP_EPSP, q)];
  d.depsp = ip[ip_index(DNL_IP_DEPSP, q)];
  d.gamma = ip[ip_index(DNL_IP_GAMMA, q)];
  d.gcum = ip[ip_index(DNL_IP_GAMMA_CUM, q)];
  d.yield = ip[ip_index(DNL_IP_YIELD, q)];
  d.T = ip[ip_index(DNL_IP_T, q)];
  d.eint = ip[ip_index(DNL_IP_EINT, q)];
  d.einel = ip[ip_index(DNL_IP_EINEL, q)];
  d.pressure = pressure;
  const double de[6] = {e0, e1, e2, e3, e4, e5};
  bool ok;
  radial_return<double>(jc, mp.twoG, mp.heatFrac, 1.0 / mp.rho0, de, dt, d, ok);
  Resolved r;
  for (int c = 0; c < 6; c++)
    r.s[c] = (float)d.s[c];
  r.kplast = (float)d.kplast;
  r.epsp = (float)d.epsp;
  r.depsp = (float)d.depsp;
  r.gamma = (float)d.gamma;
  r.gcum = (float)d.gcum;
  r.yield = (float)d.yield;
  r.T = (float)d.T;
  r.eint = (float)d.eint;
  r.einel = (float)d.einel;
  r.ok = ok;
  return r;
}

// Derivatives of the shape functions of node N at the Gauss point with local
// coordinates (xi0, xi1, xi2) (ElHex8N3D.C:561-632, ElQua4NAx.C:269-297).
template <typename R, int NPE, int N>
__device__ __forceinline__ void shape(R xi0, R xi1, R xi2, R dN[3], R &Nv)
{
  const R s0 = R(node_sign(N, 0)), s1 = R(node_sign(N, 1)), s2 = R(node_sign(N, 2));
  if constexpr (NPE == 8)
  {
    const R f0 = R(1) + s0 * xi0, f1 = R(1) + s1 * xi1, f2 = R(1) + s2 * xi2;
    dN[0] = s0 * f1 * f2 * R(0.125);
    dN[1] = s1 * f0 * f2 * R(0.125);
    dN[2] = s2 * f0 * f1 * R(0.125);
    Nv = f0 * f1 * f2 * R(0.125);
  }
  else
  {
    const R f0 = R(1) + s0 * xi0, f1 = R(1) + s1 * xi1;
    dN[0] = s0 * f1 * R(0.25);
    dN[1] = s1 * f0 * R(0.25);
    dN[2] = R(0);
    Nv = f0 * f1 * R(0.25);
  }
}

template <typename R, int NPE, int N> struct GatherJG
{
  static __device__ __forceinline__ void run(unsigned amask, int base, R xi0, R xi1, R xi2, R rx, R ry, R rz, R urx,
                                             R ury, R urz, R (&J)[3][3], R (&G)[3][3], R &Nr, R &Vr)
  {
    constexpr int DIM = (NPE == 8) ? 3 : 2;
    R dN[3], Nv;
    shape<R, NPE, N>(xi0, xi1, xi2, dN, Nv);
    const R xn[3] = {__shfl_sync(amask, rx, base + N), __shfl_sync(amask, ry, base + N),
                     DIM == 3 ? __shfl_sync(amask, rz, base + N) : R(0)};
    const R un[3] = {__shfl_sync(amask, urx, base + N), __shfl_sync(amask, ury, base + N),
                     DIM == 3 ? __shfl_sync(amask, urz, base + N) : R(0)};
#pragma unroll
    for (int i = 0; i < DIM; i++)
#pragma unroll
      for (int j = 0; j < DIM; j++)
      {
        J[i][j] += dN[j] * xn[i];
        G[i][j] += dN[j] * un[i];
      }
    if constexpr (NPE == 4)
    {
      Nr += Nv * xn[0];
      Vr += Nv * un[0];
    }
    if constexpr (N + 1 < NPE)
      GatherJG<R, NPE, N + 1>::run(amask, base, xi0, xi1, xi2, rx, ry, rz, urx, ury, urz, J, G, Nr, Vr);
  }
};

// Per-(lane, node) element forces written to shared memory for the transpose.
template <typename R, int NPE, int N> struct ForcesToShared
{
  static __device__ __forceinline__ void run(R xi0, R xi1, R xi2, const R (&P)[3][3], R hoop, R *row)
  {
    constexpr int DIM = (NPE == 8) ? 3 : 2;
    R dN[3], Nv;
    shape<R, NPE, N>(xi0, xi1, xi2, dN, Nv);
#pragma unroll
    for (int i = 0; i < DIM; i++)
    {
      R s = R(0);
#pragma unroll
      for (int k = 0; k < DIM; k++)
        s += dN[k] * P[k][i];
      if (NPE == 4 && i == 0)
        s -= Nv * hoop;
      row[N * DIM + i] = s;
    }
    if constexpr (N + 1 < NPE)
      ForcesToShared<R, NPE, N + 1>::run(xi0, xi1, xi2, P, hoop, row);
  }
};

template <int NPE> struct ElemShape
{
  static constexpr int DIM = (NPE == 8) ? 3 : 2;
  static constexpr bool AXI = (NPE == 4);
  // shared-memory row per point (padded for bank spread): the element forces
  // of the transpose, or the rotation and inverse Jacobian parked across the return
  static constexpr int ROW = (NPE * DIM > 18 ? NPE * DIM : 18) + 1;
  // the element pass's row: the rotation and J^-1 parked across the return as
  // 16-byte vectors (the hexahedron's forces need no transpose, the
  // quadrilaterals' 8 fit).  A row of 20 floats (80 B) or 22 doubles (176 B)
  // is an odd number of 16-byte units, so the 8 lanes of each phase of a
  // 16-byte access reach 8 different bank groups
  template <typename R> static constexpr int pass_row = sizeof(R) == 4 ? 20 : 22;
};

// The rotation and J^-1 of this lane's point parked in its row across the
// return: 18 values as 16-byte stores and loads (row 16-byte aligned).
template <typename R>
__device__ __forceinline__ void park_rot_inv(R *row, const R (&Rot)[9], const R (&inv)[3][3])
{
  const R v[18] = {Rot[0], Rot[1], Rot[2], Rot[3], Rot[4], Rot[5], Rot[6], Rot[7], Rot[8],
                   inv[0][0], inv[0][1], inv[0][2], inv[1][0], inv[1][1], inv[1][2], inv[2][0], inv[2][1], inv[2][2]};
  if constexpr (sizeof(R) == 4)
  {
    float4 *r4 = reinterpret_cast<float4 *>(row);
#pragma unroll
    for (int k = 0; k < 4; k++)
      r4[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
    reinterpret_cast<float2 *>(row)[8] = make_float2(v[16], v[17]);
  }
  else
  {
    double2 *r2 = reinterpret_cast<double2 *>(row);
#pragma unroll
    for (int k = 0; k < 9; k++)
      r2[k] = make_double2(v[2 * k], v[2 * k + 1]);
  }
}

template <typename R> __device__ __forceinline__ void unpark_rot_inv(const R *row, R (&Rot)[9], R (&inv)[9])
{
  R v[18];
  if constexpr (sizeof(R) == 4)
  {
    const float4 *r4 = reinterpret_cast<const float4 *>(row);
#pragma unroll
    for (int k = 0; k < 4; k++)
    {
      const float4 a = r4[k];
      v[4 * k] = a.x;
      v[4 * k + 1] = a.y;
      v[4 * k + 2] = a.z;
      v[4 * k + 3] = a.w;
    }
    const float2 b = reinterpret_cast<const float2 *>(row)[8];
    v[16] = b.x;
    v[17] = b.y;
  }
  else
  {
    const double2 *r2 = reinterpret_cast<const double2 *>(row);
#pragma unroll
    for (int k = 0; k < 9; k++)
    {
      const double2 a = r2[k];
      v[2 * k] = a.x;
      v[2 * k + 1] = a.y;
    }
  }
#pragma unroll
  for (int k = 0; k < 9; k++)
  {
    Rot[k] = v[k];
    inv[k] = v[9 + k];
  }
}

// Hexahedron in modal form.  With the node signs of node_sign(),
// s0 = -chi_3(n), s1 = -chi_2(n), s2 = -chi_4(n), s0 s1 = chi_1(n),
// s0 s2 = chi_7(n), s1 s2 = chi_6(n), s0 s1 s2 = -chi_5(n), where
// chi_w(n) = (-1)^popcount(w & n), so that the shape-function derivatives of
// ElHex8N3D.C:561-632 read
//   8 dN_n/dxi0 = -chi_3 + chi_1 xi1 + chi_7 xi2 - chi_5 xi1 xi2
//   8 dN_n/dxi1 = -chi_2 + chi_1 xi0 + chi_6 xi2 - chi_5 xi0 xi2
//   8 dN_n/dxi2 = -chi_4 + chi_7 xi0 + chi_6 xi1 - chi_5 xi0 xi1.
// The Jacobian at a Gauss point is then a combination of the Walsh sums
// W_w = sum_n chi_w(n) x_n of the element's nodes, and the nodal forces are
// the Walsh transform of the per-point terms summed over the points.  Both
// run on the element's eight lanes (lane g holds node g and Gauss point g) with
// butterflies over lane bits instead of per-node loops.

// In place: lane w of the group ends with sum_n chi_w(n) v_n.
template <typename R, int NC>
__device__ __forceinline__ void walsh8(unsigned amask, int g, R (&v)[NC])
{
#pragma unroll
  for (int k = 0; k < 3; k++)
  {
    const R sg = ((g >> k) & 1) ? R(-1) : R(1); // bit 0: v + p, bit 1: p - v
#pragma unroll
    for (int c = 0; c < NC; c++)
      v[c] = sg * v[c] + __shfl_xor_sync(amask, v[c], 1 << k);
  }
}

// The coordinates and increment of the element's first node, which every
// lane of the element subtracts: by shuffles from the element's first lane.
__device__ __forceinline__ void first_node_by_shuffle(unsigned amask, int base, const double4 &X, const double4 &U,
                                                      double4 &X0, double4 &U0)
{
  X0 = make_double4(__shfl_sync(amask, X.x, base), __shfl_sync(amask, X.y, base), __shfl_sync(amask, X.z, base), 0.0);
  U0 = make_double4(__shfl_sync(amask, U.x, base), __shfl_sync(amask, U.y, base), __shfl_sync(amask, U.z, base), 0.0);
}

// J (and G) at this lane's Gauss point from the offsets of the element's nodes
// (this lane's node offset in o[0..2] for x and o[3..5] for the increment).
// After the butterfly, lane w holds the Walsh sums W_w of the six components;
// every lane needs W_1..W_7 of each: they go through the element's shared
// memory (grp, the rows of its 8 lanes, 16-byte aligned: 48 values written,
// then read as vectors), or, without it, by register shuffles.
// The FP32 form of hex_jacobians with the element's shared rows: component i
// of the coordinates and of the increment as one packed pair (o[i], o[i+3]),
// so that the butterfly and the Jacobian rows run as paired FP32 operations
// (fma.rn.f32x2); the rows hold the pairs of Walsh index w at grp[16 i + 2 w].
__device__ __forceinline__ void hex_jacobians_paired(unsigned amask, int g, float xi0, float xi1, float xi2,
                                                     const float (&o)[6], float (&J)[3][3], float (&G)[3][3],
                                                     float *grp)
{
  float2 p[3] = {make_float2(o[0], o[3]), make_float2(o[1], o[4]), make_float2(o[2], o[5])};
#pragma unroll
  for (int k = 0; k < 3; k++)
  {
    const float sg = ((g >> k) & 1) ? -1.f : 1.f; // bit 0: v + p, bit 1: p - v
    const float2 SG = make_float2(sg, sg);
#pragma unroll
    for (int i = 0; i < 3; i++)
    {
      const float2 q = make_float2(__shfl_xor_sync(amask, p[i].x, 1 << k), __shfl_xor_sync(amask, p[i].y, 1 << k));
      p[i] = __ffma2_rn(SG, p[i], q);
    }
  }
  __syncwarp(amask); // the element's lanes are done with their rows (previous tile)
#pragma unroll
  for (int i = 0; i < 3; i++)
    reinterpret_cast<float2 *>(grp)[8 * i + g] = __fmul2_rn(p[i], make_float2(0.125f, 0.125f));
  __syncwarp(amask);
  const float2 XI0 = make_float2(xi0, xi0), XI1 = make_float2(xi1, xi1), XI2 = make_float2(xi2, xi2);
  const float2 NX01 = make_float2(-xi0 * xi1, -xi0 * xi1), NX02 = make_float2(-xi0 * xi2, -xi0 * xi2),
               NX12 = make_float2(-xi1 * xi2, -xi1 * xi2), M1 = make_float2(-1.f, -1.f);
#pragma unroll
  for (int i = 0; i < 3; i++)
  {
    const float4 *row = reinterpret_cast<const float4 *>(grp + 16 * i);
    const float4 a = row[0], b = row[1], c = row[2], d = row[3];
    const float2 w1 = make_float2(a.z, a.w), w2 = make_float2(b.x, b.y), w3 = make_float2(b.z, b.w);
    const float2 w4 = make_float2(c.x, c.y), w5 = make_float2(c.z, c.w), w6 = make_float2(d.x, d.y);
    const float2 w7 = make_float2(d.z, d.w);
    const float2 t0 = __ffma2_rn(w1, XI1, __ffma2_rn(w7, XI2, __ffma2_rn(w5, NX12, __fmul2_rn(w3, M1))));
    const float2 t1 = __ffma2_rn(w1, XI0, __ffma2_rn(w6, XI2, __ffma2_rn(w5, NX02, __fmul2_rn(w2, M1))));
    const float2 t2 = __ffma2_rn(w7, XI0, __ffma2_rn(w6, XI1, __ffma2_rn(w5, NX01, __fmul2_rn(w4, M1))));
    J[i][0] = t0.x;
    G[i][0] = t0.y;
    J[i][1] = t1.x;
    G[i][1] = t1.y;
    J[i][2] = t2.x;
    G[i][2] = t2.y;
  }
  __syncwarp(amask); // the rows are the lanes' own again from here on
}

template <typename R>
__device__ __forceinline__ void hex_jacobians(unsigned amask, int g, int base, R xi0, R xi1, R xi2, R (&o)[6],
                                              R (&J)[3][3], R (&G)[3][3], R *grp)
{
  if constexpr (sizeof(R) == 4)
    if (grp)
    {
      hex_jacobians_paired(amask, g, xi0, xi1, xi2, o, J, G, grp);
      return;
    }
  walsh8<R, 6>(amask, g, o);
#pragma unroll
  for (int c = 0; c < 6; c++)
    o[c] *= R(0.125);
  const R x01 = xi0 * xi1, x02 = xi0 * xi2, x12 = xi1 * xi2;
  if (grp)
  {
    __syncwarp(amask); // the element's lanes are done with their rows (previous tile)
#pragma unroll
    for (int c = 0; c < 6; c++)
      grp[8 * c + g] = o[c];
    __syncwarp(amask);
  }
#pragma unroll
  for (int c = 0; c < 6; c++)
  {
    R w1, w2, w3, w4, w5, w6, w7;
    if (grp)
    {
      using R4 = typename V4<R>::type;
      const R4 lo = reinterpret_cast<const R4 *>(grp + 8 * c)[0], hi = reinterpret_cast<const R4 *>(grp + 8 * c)[1];
      w1 = lo.y;
      w2 = lo.z;
      w3 = lo.w;
      w4 = hi.x;
      w5 = hi.y;
      w6 = hi.z;
      w7 = hi.w;
    }
    else
    {
      w1 = __shfl_sync(amask, o[c], base + 1);
      w2 = __shfl_sync(amask, o[c], base + 2);
      w3 = __shfl_sync(amask, o[c], base + 3);
      w4 = __shfl_sync(amask, o[c], base + 4);
      w5 = __shfl_sync(amask, o[c], base + 5);
      w6 = __shfl_sync(amask, o[c], base + 6);
      w7 = __shfl_sync(amask, o[c], base + 7);
    }
    R(&T)[3][3] = c < 3 ? J : G;
    const int i = c < 3 ? c : c - 3;
    T[i][0] = w1 * xi1 + w7 * xi2 - w5 * x12 - w3;
    T[i][1] = w1 * xi0 + w6 * xi2 - w5 * x02 - w2;
    T[i][2] = w7 * xi0 + w6 * xi1 - w5 * x01 - w4;
  }
  if (grp)
    __syncwarp(amask); // the rows are the lanes' own again from here on
}

// Nodal forces f_n = sum_g sum_k dN_n/dxi_k(xi_g) P_g[k][.] of the element,
// returned on lane n: the per-point modal terms Z_w, then a reduction over the
// eight lanes fused with the Walsh transform (at each lane bit the pair of
// lanes exchanges the half of the terms the partner keeps).
// hex_forces for components 0 and 1 as one packed FP32 pair (fma.rn.f32x2),
// the same operations as the scalar form on each.
__device__ __forceinline__ float2 hex_forces_pair(unsigned amask, int g, float xi0, float xi1, float xi2,
                                                  float2 p0, float2 p1, float2 p2)
{
  const float2 XI0 = make_float2(xi0, xi0), XI1 = make_float2(xi1, xi1), XI2 = make_float2(xi2, xi2);
  const float x01 = xi0 * xi1, x02 = xi0 * xi2, x12 = xi1 * xi2;
  const float s0 = (g & 1) ? -1.f : 1.f, s1 = (g & 2) ? -1.f : 1.f, s2 = (g & 4) ? -1.f : 1.f;
  const float2 S0 = make_float2(s0, s0), S1 = make_float2(s1, s1), S2 = make_float2(s2, s2);
  const float2 NS0 = make_float2(-s0, -s0), NS1 = make_float2(-s1, -s1), NS2 = make_float2(-s2, -s2);
  const float2 M1 = make_float2(-1.f, -1.f);
  auto shfl2 = [&](float2 v, int m) {
    return make_float2(__shfl_xor_sync(amask, v.x, m), __shfl_xor_sync(amask, v.y, m));
  };
  const float2 z1 = __ffma2_rn(XI1, p0, __fmul2_rn(XI0, p1));
  const float2 z2 = __fmul2_rn(p1, M1), z3 = __fmul2_rn(p0, M1), z4 = __fmul2_rn(p2, M1);
  const float2 z5 = __fmul2_rn(M1, __ffma2_rn(make_float2(x12, x12), p0,
                                              __ffma2_rn(make_float2(x02, x02), p1, __fmul2_rn(make_float2(x01, x01), p2))));
  const float2 z6 = __ffma2_rn(XI2, p1, __fmul2_rn(XI1, p2)), z7 = __ffma2_rn(XI2, p0, __fmul2_rn(XI0, p2));
  const float2 s0z1 = __fmul2_rn(S0, z1);
  const float2 a0 = __fadd2_rn(s0z1, __fmul2_rn(M1, shfl2(s0z1, 1)));
  const float2 a1 = __fadd2_rn(__ffma2_rn(S0, z3, z2), shfl2(__ffma2_rn(NS0, z3, z2), 1));
  const float2 a2 = __fadd2_rn(__ffma2_rn(S0, z5, z4), shfl2(__ffma2_rn(NS0, z5, z4), 1));
  const float2 a3 = __fadd2_rn(__ffma2_rn(S0, z7, z6), shfl2(__ffma2_rn(NS0, z7, z6), 1));
  const float2 b0 = __fadd2_rn(__ffma2_rn(S1, a1, a0), shfl2(__ffma2_rn(NS1, a1, a0), 2));
  const float2 b1 = __fadd2_rn(__ffma2_rn(S1, a3, a2), shfl2(__ffma2_rn(NS1, a3, a2), 2));
  return __fmul2_rn(make_float2(0.125f, 0.125f),
                    __fadd2_rn(__ffma2_rn(S2, b1, b0), shfl2(__ffma2_rn(NS2, b1, b0), 4)));
}

template <typename R>
__device__ __forceinline__ void hex_forces(unsigned amask, int g, R xi0, R xi1, R xi2, const R (&P)[3][3], R (&f)[3])
{
  if constexpr (sizeof(R) == 4)
  {
    const float2 fxy = hex_forces_pair(amask, g, xi0, xi1, xi2, make_float2(P[0][0], P[0][1]),
                                       make_float2(P[1][0], P[1][1]), make_float2(P[2][0], P[2][1]));
    f[0] = fxy.x;
    f[1] = fxy.y;
    const R x01 = xi0 * xi1, x02 = xi0 * xi2, x12 = xi1 * xi2;
    const R s0 = (g & 1) ? R(-1) : R(1), s1 = (g & 2) ? R(-1) : R(1), s2 = (g & 4) ? R(-1) : R(1);
    const R p0 = P[0][2], p1 = P[1][2], p2 = P[2][2];
    const R z1 = xi1 * p0 + xi0 * p1, z2 = -p1, z3 = -p0, z4 = -p2;
    const R z5 = -(x12 * p0 + x02 * p1 + x01 * p2);
    const R z6 = xi2 * p1 + xi1 * p2, z7 = xi2 * p0 + xi0 * p2;
    const R a0 = s0 * z1 - __shfl_xor_sync(amask, s0 * z1, 1);
    const R a1 = (z2 + s0 * z3) + __shfl_xor_sync(amask, z2 - s0 * z3, 1);
    const R a2 = (z4 + s0 * z5) + __shfl_xor_sync(amask, z4 - s0 * z5, 1);
    const R a3 = (z6 + s0 * z7) + __shfl_xor_sync(amask, z6 - s0 * z7, 1);
    const R b0 = (a0 + s1 * a1) + __shfl_xor_sync(amask, a0 - s1 * a1, 2);
    const R b1 = (a2 + s1 * a3) + __shfl_xor_sync(amask, a2 - s1 * a3, 2);
    f[2] = R(0.125) * ((b0 + s2 * b1) + __shfl_xor_sync(amask, b0 - s2 * b1, 4));
    return;
  }
  const R x01 = xi0 * xi1, x02 = xi0 * xi2, x12 = xi1 * xi2;
  const R s0 = (g & 1) ? R(-1) : R(1), s1 = (g & 2) ? R(-1) : R(1), s2 = (g & 4) ? R(-1) : R(1);
#pragma unroll
  for (int i = 0; i < 3; i++)
  {
    const R p0 = P[0][i], p1 = P[1][i], p2 = P[2][i];
    const R z1 = xi1 * p0 + xi0 * p1, z2 = -p1, z3 = -p0, z4 = -p2;
    const R z5 = -(x12 * p0 + x02 * p1 + x01 * p2);
    const R z6 = xi2 * p1 + xi1 * p2, z7 = xi2 * p0 + xi0 * p2;
    // lane bit 0: pairs (z0 = 0, z1), (z2, z3), (z4, z5), (z6, z7)
    const R a0 = s0 * z1 - __shfl_xor_sync(amask, s0 * z1, 1);
    const R a1 = (z2 + s0 * z3) + __shfl_xor_sync(amask, z2 - s0 * z3, 1);
    const R a2 = (z4 + s0 * z5) + __shfl_xor_sync(amask, z4 - s0 * z5, 1);
    const R a3 = (z6 + s0 * z7) + __shfl_xor_sync(amask, z6 - s0 * z7, 1);
    // lane bit 1: pairs (a0, a1), (a2, a3)
    const R b0 = (a0 + s1 * a1) + __shfl_xor_sync(amask, a0 - s1 * a1, 2);
    const R b1 = (a2 + s1 * a3) + __shfl_xor_sync(amask, a2 - s1 * a3, 2);
    // lane bit 2
    f[i] = R(0.125) * ((b0 + s2 * b1) + __shfl_xor_sync(amask, b0 - s2 * b1, 4));
  }
}

// The element's nodal forces from this lane's P (and hoop term), returned for
// this lane's node: modal butterflies for the hexahedron, a shared-memory
// transpose for the quadrilaterals (row: this lane's row, grp: the element's first).
template <typename R, int NPE>
__device__ __forceinline__ typename V4<R>::type element_forces(unsigned amask, int g, const R (&P)[3][3], R hoop,
                                                               R *row, R *grp)
{
  constexpr int DIM = ElemShape<NPE>::DIM;
  constexpr int ROW = ElemShape<NPE>::template pass_row<R>;
  static_assert(ROW >= NPE * DIM || NPE == 8, "the transpose needs NPE * DIM values per row");
  const R a = R(0.57735026918962576451);
  const R xi0 = R(node_sign(g, 0)) * a, xi1 = R(node_sign(g, 1)) * a, xi2 = R(node_sign(g, 2)) * a;
  typename V4<R>::type fs;
  fs.x = fs.y = fs.z = fs.w = R(0);
  if constexpr (NPE == 8)
  {
    R f[3];
    hex_forces<R>(amask, g, xi0, xi1, xi2, P, f);
    fs.x = f[0];
    fs.y = f[1];
    fs.z = f[2];
  }
  else
  {
    ForcesToShared<R, NPE, 0>::run(xi0, xi1, xi2, P, hoop, row);
    __syncwarp(amask);
#pragma unroll
    for (int l = 0; l < NPE; l++)
    {
      fs.x += grp[l * ROW + g * DIM];
      fs.y += grp[l * ROW + g * DIM + 1];
      if constexpr (DIM == 3)
        fs.z += grp[l * ROW + g * DIM + 2];
    }
  }
  return fs;
}

template <typename R, int NPE, int N> struct MassToShared
{
  static __device__ __forceinline__ void run(R xi0, R xi1, R xi2, R scale, R *row)
  {
    R dN[3], Nv;
    shape<R, NPE, N>(xi0, xi1, xi2, dN, Nv);
    row[N] = scale * Nv;
    if constexpr (N + 1 < NPE)
      MassToShared<R, NPE, N + 1>::run(xi0, xi1, xi2, scale, row);
  }
};

// ---------------------------------------------------------- element pass

#ifndef DNL_ELEM_MINB_F32
#define DNL_ELEM_MINB_F32 6
#endif
#ifndef DNL_ELEM_MINB_F64
#define DNL_ELEM_MINB_F64 4
#endif


// How the element update reaches nodes, materials and its outputs in the
// engine's own arrays (tile-major point state, node-ordered force slots).
// ONE: the model has one material, read from the kernel parameters.
template <typename R, bool ONE = false> struct EngineIo
{
  using R4 = typename V4<R>::type;
  const DevModel &M;
  int q, f0;
  __device__ __forceinline__ double4 x(int n) const { return M.x[n]; }
  __device__ __forceinline__ double4 u(int n) const { return M.u[f0][n]; }
  __device__ __forceinline__ const MatDev &mat(int e) const { return M.mat[M.emat[e]]; }
  __device__ __forceinline__ const MatDev *matp(int e) const { return M.mat + M.emat[e]; }
  __device__ __forceinline__ JC<R, ONE> law(int e) const
  {
    JC<R, ONE> j;
    if constexpr (ONE)
      j.q = one_params<R>(M);
    else
      j.load(mat(e));
    return j;
  }
  __device__ __forceinline__ double rho0(int e) const
  {
    if constexpr (ONE)
      return M.one_rho0;
    else
      return mat(e).rho0;
  }
  __device__ __forceinline__ void put(int c, R v) const { ipw<R>(M, c, q, v); }
  __device__ __forceinline__ void slot(const R4 &v) const { reinterpret_cast<R4 *>(M.slot)[M.slot_pos[q]] = v; }
  __device__ __forceinline__ const float *ip32() const { return reinterpret_cast<const float *>(M.ip); }
  __device__ __forceinline__ void first_node(unsigned amask, int base, const double4 &X, const double4 &U,
                                             double4 &X0, double4 &U0) const
  {
    first_node_by_shuffle(amask, base, X, U, X0, U0);
  }
};

// Where the element update reads the old point state from: global memory, or
// the tile staged in shared memory by the bulk copies.
template <typename R> struct GlobalState
{
  const DevModel &M;
  int q;
  __device__ __forceinline__ R operator()(int c) const { return ipv<R>(M, c, q); }
};
template <typename R> struct SharedTile
{
  const R *buf;
  int t;
  // a staged tile holds the first DNL_IP_NREAD runs (the pass never reads the others)
  __device__ __forceinline__ R operator()(int c) const { return buf[ip_slot(c) * TILE + t]; }
};

// Jacobian J = sum x_n dN_n/dxi and G = sum du_n dN_n/dxi at this lane's Gauss
// point from the element's nodes (lane g holds node g), then detJ, J^-1 and the
// displacement gradient H = F - I = G J^-1 (+ the axisymmetric hoop term
// F33 - 1 = sum N_n du_r,n / r, ElementAxi.C:78-100).
// grp: the element's shared-memory rows (16-byte aligned, at least 48
// values), or nullptr: see hex_jacobians.  X0, U0: the element's first node.
template <typename R, int NPE>
__device__ __forceinline__ void kinematics(unsigned amask, int g, int base, const double4 &X, const double4 &U,
                                           const double4 &X0, const double4 &U0, R &detJ, R (&inv)[3][3], R &radius,
                                           R (&H)[9], bool axi, R *grp)
{
  constexpr int DIM = ElemShape<NPE>::DIM;
  const bool AXI = ElemShape<NPE>::AXI && axi;
  const double x0 = X0.x, y0 = X0.y, z0 = X0.z;
  const double ux0 = U0.x, uy0 = U0.y, uz0 = U0.z;
  // element-local offsets keep the FP32 path free of large-coordinate cancellation
  const R rx = R(X.x - x0), ry = R(X.y - y0), rz = R(X.z - z0);
  const R urx = R(U.x - ux0), ury = R(U.y - uy0), urz = R(U.z - uz0);
  const R a = R(0.57735026918962576451); // 1/sqrt(3)
  const R xi0 = R(node_sign(g, 0)) * a, xi1 = R(node_sign(g, 1)) * a, xi2 = R(node_sign(g, 2)) * a;
  R J[3][3], G[3][3];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
      J[i][j] = G[i][j] = R(0);
  R Nr = R(0), Vr = R(0);
  if constexpr (NPE == 8)
  {
    R o[6] = {rx, ry, rz, urx, ury, urz};
    hex_jacobians<R>(amask, g, base, xi0, xi1, xi2, o, J, G, grp);
  }
  else
    GatherJG<R, NPE, 0>::run(amask, base, xi0, xi1, xi2, rx, ry, rz, urx, ury, urz, J, G, Nr, Vr);
  radius = R(1);
  if (AXI)
  {
    // r = sum N_n x_n (ElementAxi.C:46-59) and sum N_n du_n, from the offsets
    radius = R(x0 + (double)Nr);
    Vr += R(ux0);
  }
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
      inv[i][j] = R(0);
  if constexpr (DIM == 2)
  {
    detJ = J[0][0] * J[1][1] - J[1][0] * J[0][1];
    const R id = R(1) / detJ;
    inv[0][0] = J[1][1] * id;
    inv[0][1] = -J[0][1] * id;
    inv[1][0] = -J[1][0] * id;
    inv[1][1] = J[0][0] * id;
  }
  else
  {
    const R c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    const R c01 = J[0][2] * J[2][1] - J[0][1] * J[2][2];
    const R c02 = J[0][1] * J[1][2] - J[0][2] * J[1][1];
    detJ = J[0][0] * c00 + J[1][0] * c01 + J[2][0] * c02;
    const R id = R(1) / detJ;
    inv[0][0] = c00 * id;
    inv[0][1] = c01 * id;
    inv[0][2] = c02 * id;
    inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) * id;
    inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
    inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
    inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) * id;
    inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
    inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
  }
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
    {
      R s = R(0);
#pragma unroll
      for (int k = 0; k < DIM; k++)
        s += G[i][k] * inv[k][j];
      H[3 * i + j] = (i < DIM && j < DIM) ? s : R(0);
    }
  if (AXI)
    H[8] = Vr / radius;
}

// One increment's work at one Gauss point (Explicit.C:204-226 + the density of
// Explicit::computeDensity; Element.C:1103-1256 with the Jacobian of
// ElementPlane.C:46-102 / Element3D.C:64-115 on the current coordinates):
// strain increment and rotation by polar decomposition, element-mean pressure,
// radial return, final rotation, density, and the element's nodal forces,
// summed over its points through shared memory and stored in node order.
// `row` is this lane's shared-memory row, `grp` the row of the element's first lane.
// The element-pass modes run the same update split in two (element_front /
// element_back below); this single body is what the plain variants use (the
// split costs the plain variants about 10 % in spilled registers).
template <typename R, int NPE, class Src, class Io>
__device__ __forceinline__ void element_update(const Io &io, Ctl *C, int q, int e, int g, int base, unsigned amask,
                                               int node, const Src &old, R *row, R *grp)
{
  constexpr int DIM = ElemShape<NPE>::DIM;
  const bool AXI = ElemShape<NPE>::AXI && !(C->plane);
  using R4 = typename V4<R>::type;
  const double dt = C->dt_eff;
  const double4 X = io.x(node);
  const double4 U = io.u(node);
  double4 X0, U0;
  io.first_node(amask, base, X, U, X0, U0);

  R detJ, inv[3][3], radius, dE[6], Rot[9];
  {
    R H[9];
    kinematics<R, NPE>(amask, g, base, X, U, X0, U0, detJ, inv, radius, H, !C->plane, grp);
    polar_lnU<R>(H, dE, Rot);
  }
  if (detJ < R(0))
    raise_status(C, DNL_ERR_NEG_JACOBIAN, e);
  R WxdJ = detJ; // Gauss weight 1
  if (AXI)
    WxdJ *= R(6.28318530717958647692) * radius;

  // element-mean volumetric increment (Element::computePressure, Element.C:1125-1143)
  const R trSum = group_sum<NPE>(amask, dE[0] + dE[3] + dE[5]);

  // total strain: Strain += dE, then the final rotation (Element.C:1116-1161)
  {
    R strain[6];
#pragma unroll
    for (int c = 0; c < 6; c++)
      strain[c] = old(DNL_IP_STRAIN + c) + dE[c];
    rotate_sym<R>(Rot, strain);
#pragma unroll
    for (int c = 0; c < 6; c++)
      io.put(DNL_IP_STRAIN + c, strain[c]);
  }

  // the rotation and J^-1 wait in shared memory while the return holds its registers
  park_rot_inv<R>(row, Rot, inv);

  // J2 radial return with Johnson-Cook hardening (Element.C:407-622)
  ReturnState<R> st;
#pragma unroll
  for (int c = 0; c < 6; c++)
    st.s[c] = old(DNL_IP_STRESS + c);
  st.epsp = old(DNL_IP_EPSP);
  st.depsp = old(DNL_IP_DEPSP);
  st.gamma = old(DNL_IP_GAMMA);
  st.gcum = old(DNL_IP_GAMMA_CUM);
  st.yield = old(DNL_IP_YIELD);
  st.T = old(DNL_IP_T);
  st.eint = old(DNL_IP_EINT);
  st.einel = old(DNL_IP_EINEL);
  const auto jc = io.law(e);
  st.pressure = (st.s[0] + st.s[3] + st.s[5]) / R(3) + jc.K() * (trSum / R(NPE));
  {
    bool ok;
    radial_return<R>(jc, jc.twoG(), jc.heatFrac(), jc.invRho0(), dE, R(dt), st, ok, R(-1), C->direct != 0);
    if (!ok)
    {
      if constexpr (sizeof(R) == 4)
      {
        atomicAdd(&C->resolves, 1);
        const Resolved r = resolve_fp64(io.ip32(), q, io.matp(e), dE[0], dE[1], dE[2], dE[3], dE[4], dE[5], dt,
                                        st.pressure);
        if (!r.ok)
          raise_status(C, DNL_ERR_NEWTON, q);
#pragma unroll
        for (int c = 0; c < 6; c++)
          st.s[c] = r.s[c];
        st.kplast = r.kplast;
        st.epsp = r.epsp;
        st.depsp = r.depsp;
        st.gamma = r.gamma;
        st.gcum = r.gcum;
        st.yield = r.yield;
        st.T = r.T;
        st.eint = r.eint;
        st.einel = r.einel;
      }
      else
        raise_status(C, DNL_ERR_NEWTON, q);
    }
  }

  // final rotation of the plastic strain (PlasticStrain += gamma s*/|s*|,
  // Element.C:587) and of the stress, state write-back
  R iv[9]; // J^-1, row-major
  unpark_rot_inv<R>(row, Rot, iv);
  {
    R ep[6];
    const R pn = (st.s[0] + st.s[3] + st.s[5]) / R(3);
#pragma unroll
    for (int c = 0; c < 6; c++)
      ep[c] = old(DNL_IP_PLASTIC_STRAIN + c) + st.kplast * (st.s[c] - ((c == 0 || c == 3 || c == 5) ? pn : R(0)));
    rotate_sym2<R>(Rot, ep, st.s);
#pragma unroll
    for (int c = 0; c < 6; c++)
      io.put(DNL_IP_PLASTIC_STRAIN + c, ep[c]);
  }
  R rho = R(io.rho0(e)) * old(DNL_IP_DETJ0) / detJ; // Element::computeDensity (Element.C:1243-1256)
  if (AXI)
    rho /= radius;
#pragma unroll
  for (int c = 0; c < 6; c++)
    io.put(DNL_IP_STRESS + c, st.s[c]);
  io.put(DNL_IP_EPSP, st.epsp);
  io.put(DNL_IP_DEPSP, st.depsp);
  io.put(DNL_IP_GAMMA, st.gamma);
  io.put(DNL_IP_GAMMA_CUM, st.gcum);
  io.put(DNL_IP_YIELD, st.yield);
  io.put(DNL_IP_T, st.T);
  io.put(DNL_IP_PRESSURE, st.pressure);
  io.put(DNL_IP_EINT, st.eint);
  io.put(DNL_IP_EINEL, st.einel);
  io.put(DNL_IP_DENSITY, rho);

  // internal forces f_n = -sum_g dN_n/dx . sigma w detJ (Element.C:362-404):
  // with P = -w detJ J^-1 sigma, f_n,i = sum_k dN_n/dxi_k P_ki
  R P[3][3];
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int i = 0; i < 3; i++)
    {
      R s = R(0);
#pragma unroll
      for (int j = 0; j < DIM; j++)
        s += iv[3 * k + j] * st.s[sym_index(j, i)];
      P[k][i] = -WxdJ * s;
    }
  const R hoop = AXI ? st.s[5] / radius * WxdJ : R(0);
  io.slot(element_forces<R, NPE>(amask, g, P, hoop, row, grp));
}

// What the first half of an element update hands to the second: the strain
// increment, the Jacobian terms and the point state loaded for the return (the
// rotation and J^-1 wait in the lane's shared-memory row).
template <typename R> struct Front
{
  R detJ, WxdJ, radius;
  R dE[6];
  ReturnState<R> st;
};

// The element update of element_update above in two halves, for the
// element-pass modes: element_front runs up to the start of the return,
// element_back from the return on; the mode kernel runs block-wide work (the
// learned guess) in between.  Same arithmetic as element_update.
template <typename R, int NPE, class Src, class Io>
__device__ __forceinline__ void element_front(const Io &io, Ctl *C, int e, int g, int base, unsigned amask, int node,
                                              const Src &old, R *row, R *grp, Front<R> &f)
{
  const bool AXI = ElemShape<NPE>::AXI && !(C->plane);
  const MatDev &mp = io.mat(e);
  const double4 X = io.x(node);
  const double4 U = io.u(node);
  double4 X0, U0;
  io.first_node(amask, base, X, U, X0, U0);

  R inv[3][3], Rot[9];
  {
    R H[9];
    kinematics<R, NPE>(amask, g, base, X, U, X0, U0, f.detJ, inv, f.radius, H, !C->plane, grp);
    polar_lnU<R>(H, f.dE, Rot);
  }
  if (f.detJ < R(0))
    raise_status(C, DNL_ERR_NEG_JACOBIAN, e);
  f.WxdJ = f.detJ; // Gauss weight 1
  if (AXI)
    f.WxdJ *= R(6.28318530717958647692) * f.radius;

  // element-mean volumetric increment (Element::computePressure, Element.C:1125-1143)
  const R trSum = group_sum<NPE>(amask, f.dE[0] + f.dE[3] + f.dE[5]);

  // total strain: Strain += dE, then the final rotation (Element.C:1116-1161)
  {
    R strain[6];
#pragma unroll
    for (int c = 0; c < 6; c++)
      strain[c] = old(DNL_IP_STRAIN + c) + f.dE[c];
    rotate_sym<R>(Rot, strain);
#pragma unroll
    for (int c = 0; c < 6; c++)
      io.put(DNL_IP_STRAIN + c, strain[c]);
  }

  // the rotation and J^-1 wait in shared memory while the return holds its registers
  park_rot_inv<R>(row, Rot, inv);

  ReturnState<R> &st = f.st;
#pragma unroll
  for (int c = 0; c < 6; c++)
    st.s[c] = old(DNL_IP_STRESS + c);
  st.epsp = old(DNL_IP_EPSP);
  st.depsp = old(DNL_IP_DEPSP);
  st.gamma = old(DNL_IP_GAMMA);
  st.gcum = old(DNL_IP_GAMMA_CUM);
  st.yield = old(DNL_IP_YIELD);
  st.T = old(DNL_IP_T);
  st.eint = old(DNL_IP_EINT);
  st.einel = old(DNL_IP_EINEL);
  st.pressure = (st.s[0] + st.s[3] + st.s[5]) / R(3) + R(mp.K) * (trSum / R(NPE));
}

// Second half: J2 radial return with Johnson-Cook hardening (Element.C:407-622)
// from gamma0 (< 0: the reference's warm start), final rotation, density,
// write-back and the element forces.  Returns the yield-function evaluations
// of the return (0 for an elastic point).
template <typename R, int NPE, class Src, class Io>
__device__ __forceinline__ int element_back(const Io &io, Ctl *C, int q, int e, int g, unsigned amask,
                                            const Src &old, R *row, R *grp, Front<R> &f, R gamma0 = R(-1))
{
  constexpr int DIM = ElemShape<NPE>::DIM;
  const bool AXI = ElemShape<NPE>::AXI && !(C->plane);
  using R4 = typename V4<R>::type;
  const double dt = C->dt_eff;
  const MatDev &mp = io.mat(e);
  ReturnState<R> &st = f.st;
  const R *dE = f.dE;
  int iters;
  {
    JC<R> jc;
    jc.load(mp);
    bool ok;
    iters = radial_return<R>(jc, R(mp.twoG), R(mp.heatFrac), R(1.0 / mp.rho0), dE, R(dt), st, ok, gamma0,
                             C->direct != 0);
    if (!ok)
    {
      if constexpr (sizeof(R) == 4)
      {
        atomicAdd(&C->resolves, 1);
        const Resolved r = resolve_fp64(io.ip32(), q, io.matp(e), dE[0], dE[1], dE[2], dE[3], dE[4], dE[5], dt,
                                        st.pressure);
        if (!r.ok)
          raise_status(C, DNL_ERR_NEWTON, q);
#pragma unroll
        for (int c = 0; c < 6; c++)
          st.s[c] = r.s[c];
        st.kplast = r.kplast;
        st.epsp = r.epsp;
        st.depsp = r.depsp;
        st.gamma = r.gamma;
        st.gcum = r.gcum;
        st.yield = r.yield;
        st.T = r.T;
        st.eint = r.eint;
        st.einel = r.einel;
      }
      else
        raise_status(C, DNL_ERR_NEWTON, q);
    }
  }

  // final rotation of the plastic strain (PlasticStrain += gamma s*/|s*|,
  // Element.C:587) and of the stress, state write-back
  R Rot[9], iv[9]; // iv: J^-1, row-major
  unpark_rot_inv<R>(row, Rot, iv);
  {
    R ep[6];
    const R pn = (st.s[0] + st.s[3] + st.s[5]) / R(3);
#pragma unroll
    for (int c = 0; c < 6; c++)
      ep[c] = old(DNL_IP_PLASTIC_STRAIN + c) + st.kplast * (st.s[c] - ((c == 0 || c == 3 || c == 5) ? pn : R(0)));
    rotate_sym2<R>(Rot, ep, st.s);
#pragma unroll
    for (int c = 0; c < 6; c++)
      io.put(DNL_IP_PLASTIC_STRAIN + c, ep[c]);
  }
  R rho = R(mp.rho0) * old(DNL_IP_DETJ0) / f.detJ; // Element::computeDensity (Element.C:1243-1256)
  if (AXI)
    rho /= f.radius;
#pragma unroll
  for (int c = 0; c < 6; c++)
    io.put(DNL_IP_STRESS + c, st.s[c]);
  io.put(DNL_IP_EPSP, st.epsp);
  io.put(DNL_IP_DEPSP, st.depsp);
  io.put(DNL_IP_GAMMA, st.gamma);
  io.put(DNL_IP_GAMMA_CUM, st.gcum);
  io.put(DNL_IP_YIELD, st.yield);
  io.put(DNL_IP_T, st.T);
  io.put(DNL_IP_PRESSURE, st.pressure);
  io.put(DNL_IP_EINT, st.eint);
  io.put(DNL_IP_EINEL, st.einel);
  io.put(DNL_IP_DENSITY, rho);

  // internal forces f_n = -sum_g dN_n/dx . sigma w detJ (Element.C:362-404):
  // with P = -w detJ J^-1 sigma, f_n,i = sum_k dN_n/dxi_k P_ki
  R P[3][3];
#pragma unroll
  for (int k = 0; k < 3; k++)
#pragma unroll
    for (int i = 0; i < 3; i++)
    {
      R s = R(0);
#pragma unroll
      for (int j = 0; j < DIM; j++)
        s += iv[3 * k + j] * st.s[sym_index(j, i)];
      P[k][i] = -f.WxdJ * s;
    }
  const R hoop = AXI ? st.s[5] / f.radius * f.WxdJ : R(0);
  io.slot(element_forces<R, NPE>(amask, g, P, hoop, row, grp));
  return iters;
}

// Start of the solve: reference Jacobian detJ0 (ElementPlane.C:96-100,
// Element3D.C:111-112), initial point state (Element::initializeData,
// Element.C:258-301) and the element lumped masses (Element::computeMassMatrix,
// Element.C:304-339) into the slots.  One thread per Gauss point.
template <typename R, int NPE>
__global__ void __launch_bounds__(TILE) k_element_start(DevModel M)
{
  constexpr int ROW = ElemShape<NPE>::ROW;
  using R4 = typename V4<R>::type;
  __shared__ __align__(16) R sh[TILE * ROW];
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const int g = lane & (NPE - 1);
  const int base = lane & ~(NPE - 1);
  const int e = q / NPE;
  const bool act = e < M.nE;
  const unsigned amask = __ballot_sync(0xffffffffu, act);
  if (!act)
    return;
  const int inst = (M.nInst > 1) ? find_segment(M.inst_elem_begin, M.nInst, e) : 0;
  const bool AXI = ElemShape<NPE>::AXI && !M.ctl[inst].plane;
  const MatDev &mp = M.mat[M.emat[e]];
  const int node = M.conn[q];
  R detJ, inv[3][3], radius, H[9];
  const double4 X = M.x[node], U = make_double4(0, 0, 0, 0);
  double4 X0, U0;
  first_node_by_shuffle(amask, base, X, U, X0, U0);
  kinematics<R, NPE>(amask, g, base, X, U, X0, U0, detJ, inv, radius, H, !M.ctl[inst].plane,
                     (R *)nullptr);
  if (detJ < R(0))
    raise_status(M.ctl + inst, DNL_ERR_NEG_JACOBIAN, e);
  R WxdJ = detJ;
  if (AXI)
    WxdJ *= R(6.28318530717958647692) * radius;
  const R rho0 = R(mp.rho0);
#pragma unroll
  for (int c = 0; c < DNL_IP_DETJ0; c++)
    ipw<R>(M, c, q, R(0));
  ipw<R>(M, DNL_IP_DETJ0, q, AXI ? detJ * radius : detJ);
  ipw<R>(M, DNL_IP_T, q, R(mp.T0));
  ipw<R>(M, DNL_IP_DENSITY, q, rho0);
  const R a = R(0.57735026918962576451);
  R *row = sh + threadIdx.x * ROW, *grp = sh + (threadIdx.x - g) * ROW;
  MassToShared<R, NPE, 0>::run(R(node_sign(g, 0)) * a, R(node_sign(g, 1)) * a, R(node_sign(g, 2)) * a,
                               rho0 * WxdJ, row);
  __syncwarp(amask);
  R m = R(0);
#pragma unroll
  for (int l = 0; l < NPE; l++)
    m += grp[l * ROW + g];
  R4 s;
  s.x = m;
  s.y = s.z = s.w = R(0);
  reinterpret_cast<R4 *>(M.slot)[M.slot_pos[q]] = s;
}

// ------------------------------------------------------ batch work lists

// Tiles of TILE points that hold points of instance c's elements (the first
// and last may be shared with the neighbouring instances).
__device__ __forceinline__ int instance_tiles(const Ctl &c, int npe)
{
  return (c.elem_end * npe + TILE - 1) / TILE - (c.elem_begin * npe) / TILE;
}

// One block: the list of the instances that run this increment and the
// prefix sums of their tiles, nodes and elements, so that the passes of a
// batch spread only the running instances' work over the GPU (a batch ends
// with a few long-running instances among hundreds that have stopped).
__global__ void __launch_bounds__(1024) k_active_list(DevModel M, int npe)
{
  __shared__ int wsum[6][32];
  __shared__ int carry[6];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  if (t < 6)
    carry[t] = 0;
  __syncthreads();
  for (int base = 0; base < M.nInst; base += 1024)
  {
    const int i = base + t;
    // running, tiles, nodes, elements; running with the time step due, its elements
    int v[6] = {0, 0, 0, 0, 0, 0};
    if (i < M.nInst)
    {
      const Ctl &c = M.ctl[i];
      if (c.active)
      {
        v[0] = 1;
        v[1] = instance_tiles(c, npe);
        v[2] = c.node_end - c.node_begin;
        v[3] = c.elem_end - c.elem_begin;
        if (c.due)
        {
          v[4] = 1;
          v[5] = v[3];
        }
      }
    }
    int inc[6];
#pragma unroll
    for (int k = 0; k < 6; k++)
    {
      inc[k] = v[k];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1)
      {
        const int y = __shfl_up_sync(0xffffffffu, inc[k], o);
        if (lane >= o)
          inc[k] += y;
      }
      if (lane == 31)
        wsum[k][w] = inc[k];
    }
    __syncthreads();
    if (w == 0)
    {
#pragma unroll
      for (int k = 0; k < 6; k++)
      {
        int x = wsum[k][lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
        {
          const int y = __shfl_up_sync(0xffffffffu, x, o);
          if (lane >= o)
            x += y;
        }
        wsum[k][lane] = x; // inclusive over the warps
      }
    }
    __syncthreads();
    int ex[6];
#pragma unroll
    for (int k = 0; k < 6; k++)
      ex[k] = carry[k] + inc[k] - v[k] + (w > 0 ? wsum[k][w - 1] : 0);
    if (v[0])
    {
      M.act_list[ex[0]] = i;
      M.act_tile_pre[ex[0]] = ex[1];
      M.act_node_pre[ex[0]] = ex[2];
      M.act_elem_pre[ex[0]] = ex[3];
    }
    if (v[4])
    {
      M.due_list[ex[4]] = i;
      M.due_elem_pre[ex[4]] = ex[5];
    }
    __syncthreads();
    if (t < 6)
      carry[t] += wsum[t][31];
    __syncthreads();
  }
  if (t == 0)
  {
    *M.act_count = carry[0];
    M.act_tile_pre[carry[0]] = carry[1];
    M.act_node_pre[carry[0]] = carry[2];
    M.act_elem_pre[carry[0]] = carry[3];
    *M.due_count = carry[4];
    M.due_elem_pre[carry[4]] = carry[5];
  }
}

// Work slots of the element pass.  A single model: one slot per tile while it
// runs.  A batch: the tiles of the running instances (k_active_list); a tile
// shared by two running instances is a slot of each, and each pass updates
// only its own instance's elements (their points and slots are disjoint).
template <int NPE> struct TileMap
{
  const DevModel &M;
  int nTiles;
  __device__ __forceinline__ int count() const
  {
    if (M.nInst == 1)
      return M.ctl[0].active ? nTiles : 0;
    return M.act_tile_pre[*M.act_count];
  }
  __device__ __forceinline__ void get(int slot, int &tile, int &inst) const
  {
    if (M.nInst == 1)
    {
      tile = slot;
      inst = 0;
      return;
    }
    const int a = find_segment(M.act_tile_pre, *M.act_count, slot);
    inst = M.act_list[a];
    tile = (M.ctl[inst].elem_begin * NPE) / TILE + (slot - M.act_tile_pre[a]);
  }
};

// Element pass, one thread per Gauss point, state read straight from global memory.
// One block per work slot (TileMap): a tile of a single model, or a tile of a
// running instance of a batch (blocks past the slots leave at once).  The
// same binary serves both, so that a model gives the same bits alone and in a
// batch; the persistent variants below are the ones that suit the tail of a
// batch, where few instances still run.
// PTS points per block: TILE (a block per work slot), 2 TILE (two slots per
// block) or TILE / 2 (two blocks per slot); MINB blocks of PTS threads per SM.
template <typename R, int NPE, int MINB, int PTS = TILE, bool ONE = false>
__global__ void __launch_bounds__(PTS, MINB) k_element(DevModel M, int nTiles)
{
  static_assert(PTS == TILE || PTS == 2 * TILE || 2 * PTS == TILE, "PTS: half, one or two tiles");
  pdl_wait();
  constexpr int ROW = ElemShape<NPE>::template pass_row<R>;
  __shared__ __align__(16) R sh[PTS * ROW];
  const int lane = threadIdx.x & 31;
  const int g = lane & (NPE - 1);
  const int base = lane & ~(NPE - 1);
  const TileMap<NPE> map{M, nTiles};
  const int slot = PTS >= TILE ? (int)(blockIdx.x * (PTS / TILE) + threadIdx.x / TILE) : (int)(blockIdx.x / 2);
  if (slot >= map.count())
    return;
  int tile, inst;
  map.get(slot, tile, inst);
  const int t = PTS >= TILE ? (int)(threadIdx.x % TILE) : (int)((blockIdx.x % 2) * PTS + threadIdx.x);
  const int q = tile * TILE + t;
  const int e = q / NPE;
  Ctl *C = M.ctl + inst;
  const bool act = e >= C->elem_begin && e < C->elem_end && C->active;
  const unsigned amask = __ballot_sync(0xffffffffu, act);
  if (!act)
    return;
  GlobalState<R> old{M, q};
  EngineIo<R, ONE> io{M, q, C->f0};
  element_update<R, NPE>(io, C, q, e, g, base, amask, M.conn[q], old, sh + threadIdx.x * ROW,
                         sh + (threadIdx.x - g) * ROW);
}

// ----------------------------------------------- bulk-copy (TMA) primitives

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// global -> shared bulk copy completing on an mbarrier (no multicast)
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// the same with an evict-first L2 policy: for the point state, which is read
// once per increment (see ipv)
__device__ __forceinline__ void bulk_g2s_ef(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
  uint32_t ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
               : "=r"(ok)
               : "r"(smem_u32(bar)), "r"(parity)
               : "memory");
  return ok != 0;
}

// Bounded wait for the phase `parity` of an mbarrier (bulk copies, tensor-core
// commits); false when it did not complete within about two seconds of SM
// clock (the caller flags an error and goes on without the data).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
  const long long start = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - start > (1ll << 32))
      return false;
  return true;
}

#include "dnl_mlp.cuh"

// Element pass as a persistent kernel over tiles of TILE Gauss points: while a
// block computes one tile, the bulk-copy engine brings the next tile's point
// state (one contiguous block in the tile-major layout) and connectivity into
// the other shared-memory buffer.  Results go straight to global memory.
template <typename R, int NPE, int MINB, bool ONE = false>
__global__ void __launch_bounds__(TILE, MINB) k_element_tma(DevModel M, int nTiles, int *err)
{
  pdl_wait();
  constexpr int ROW = ElemShape<NPE>::template pass_row<R>;
  constexpr uint32_t STATE_BYTES = DNL_IP_NREAD * TILE * sizeof(R); // the runs the pass reads
  constexpr uint32_t CONN_BYTES = TILE * sizeof(int);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  R *state[2] = {reinterpret_cast<R *>(smem_raw), reinterpret_cast<R *>(smem_raw + STATE_BYTES)};
  int *conn[2] = {reinterpret_cast<int *>(smem_raw + 2 * STATE_BYTES),
                  reinterpret_cast<int *>(smem_raw + 2 * STATE_BYTES + CONN_BYTES)};
  R *rows = reinterpret_cast<R *>(smem_raw + 2 * STATE_BYTES + 2 * CONN_BYTES);
  __shared__ __align__(8) uint64_t bar[2];
  const int t = threadIdx.x;
  const int lane = t & 31;
  const int g = lane & (NPE - 1);
  const int base = lane & ~(NPE - 1);
  if (t == 0)
  {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto issue = [&](int tile, int b) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&bar[b], STATE_BYTES + CONN_BYTES);
    bulk_g2s_ef(state[b], reinterpret_cast<const R *>(M.ip) + (size_t)tile * DNL_IP_NCOMP * TILE, STATE_BYTES, &bar[b]);
    bulk_g2s(conn[b], M.conn + (size_t)tile * TILE, CONN_BYTES, &bar[b]);
  };
  // Work slots (TileMap): the tiles of the running instances only.  The
  // running set does not change during the pass, so every thread of the
  // block walks the same sequence.
  const TileMap<NPE> map{M, nTiles};
  const int nSlots = map.count();
  int slot = blockIdx.x, tile = 0, inst = 0, ntile = 0, ninst = 0;
  if (slot < nSlots)
    map.get(slot, tile, inst);
  if (t == 0 && slot < nSlots)
    issue(tile, 0);
  uint32_t phase[2] = {0, 0};
  for (int b = 0; slot < nSlots; slot += gridDim.x, tile = ntile, inst = ninst, b ^= 1)
  {
    const bool more = slot + (int)gridDim.x < nSlots;
    if (more)
      map.get(slot + gridDim.x, ntile, ninst);
    if (t == 0 && more)
      issue(ntile, b ^ 1);
    if (!mbar_wait(&bar[b], phase[b]))
    {
      atomicExch(err, 1);
      mbar_wait(&bar[b], phase[b]);
      return;
    }
    phase[b] ^= 1;
    const int q = tile * TILE + t;
    const int e = q / NPE;
    Ctl *C = M.ctl + inst;
    const bool act = e >= C->elem_begin && e < C->elem_end && C->active;
    const unsigned amask = __ballot_sync(0xffffffffu, act);
    if (act)
    {
      SharedTile<R> old{state[b], t};
      EngineIo<R, ONE> io{M, q, C->f0};
      element_update<R, NPE>(io, C, q, e, g, base, amask, conn[b][t], old, rows + t * ROW, rows + (t - g) * ROW);
    }
    __syncthreads(); // the buffer is refilled two tiles later
  }
}

// ------------------------------------- element pass with staged node data

// 16-byte asynchronous global -> shared copies (no mbarrier), grouped per tile
__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src)
{
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Element update I/O for a tile whose node coordinates and increments, force
// slot positions and element materials were staged in shared memory.
// A staged node vector: x and y in one 16-byte run, z in another array, so
// that a tile of nodes takes 24 bytes a node (the device arrays are double4).
struct StagedVec
{
  const double2 *xy;
  const double *z;
  __device__ __forceinline__ double4 get(int back = 0) const
  {
    const double2 a = xy[-back];
    return make_double4(a.x, a.y, z[-back], 0.0);
  }
};

template <typename R, bool ONE = false> struct StagedIo
{
  using R4 = typename V4<R>::type;
  const DevModel &M;
  int q;
  StagedVec nx, nu; // this lane's node
  int spos;
  const MatDev *mp;
  int g; // this lane's place in its element
  __device__ __forceinline__ double4 x(int) const { return nx.get(); }
  __device__ __forceinline__ double4 u(int) const { return nu.get(); }
  __device__ __forceinline__ const MatDev &mat(int) const { return *mp; }
  __device__ __forceinline__ const MatDev *matp(int) const { return mp; }
  __device__ __forceinline__ JC<R, ONE> law(int) const
  {
    JC<R, ONE> j;
    if constexpr (ONE)
      j.q = one_params<R>(M);
    else
      j.load(*mp);
    return j;
  }
  __device__ __forceinline__ double rho0(int) const
  {
    if constexpr (ONE)
      return M.one_rho0;
    else
      return mp->rho0;
  }
  __device__ __forceinline__ void put(int c, R v) const { ipw<R>(M, c, q, v); }
  __device__ __forceinline__ void slot(const R4 &v) const { reinterpret_cast<R4 *>(M.slot)[spos] = v; }
  __device__ __forceinline__ const float *ip32() const { return reinterpret_cast<const float *>(M.ip); }
  // the element's first node is staged g entries before this lane's
  __device__ __forceinline__ void first_node(unsigned, int, const double4 &, const double4 &, double4 &X0,
                                             double4 &U0) const
  {
    X0 = nx.get(g);
    U0 = nu.get(g);
  }
};

// Element pass as a persistent kernel with three pipelines a tile apart: the
// point state, force-slot positions and element materials of the next tile
// come by bulk copy (mbarrier), the connectivity two tiles ahead, and the
// coordinates and increments of the next tile's nodes are gathered by
// asynchronous copies while the current tile computes, so the update reads
// every input from shared memory.
template <typename R, int NPE> struct StageLayout
{
  static constexpr int EPT = TILE / NPE; // elements per tile
  static constexpr uint32_t STATE_BYTES = DNL_IP_NREAD * TILE * sizeof(R); // the runs the pass reads
  // coordinates then increments, each as xy[TILE] (double2) and z[TILE]
  static constexpr uint32_t NODE_BYTES = 2 * TILE * (sizeof(double2) + sizeof(double));
  static constexpr uint32_t IDX_BYTES = TILE * sizeof(int);
  static constexpr uint32_t EMAT_BYTES = EPT * sizeof(int);
  static_assert(EMAT_BYTES % 16 == 0, "bulk copies move multiples of 16 bytes");
  // shared memory: state[2] | nodes[2] | (slot positions, materials)[2] | connectivity[3] | rows
  static constexpr uint32_t OFF_NODES = 2 * STATE_BYTES;
  static constexpr uint32_t OFF_IDX = OFF_NODES + 2 * NODE_BYTES;
  static constexpr uint32_t IDX_STRIDE = IDX_BYTES + EMAT_BYTES;
  static constexpr uint32_t OFF_CONN = OFF_IDX + 2 * IDX_STRIDE;
  static constexpr uint32_t OFF_ROWS = OFF_CONN + 3 * IDX_BYTES;
  static constexpr uint32_t BYTES = OFF_ROWS + TILE * ElemShape<NPE>::template pass_row<R> * sizeof(R);
};

template <typename R, int NPE, int MINB, bool ONE = false>
__global__ void __launch_bounds__(TILE, MINB) k_element_stage(DevModel M, int nTiles, int *err)
{
  pdl_wait();
  using L = StageLayout<R, NPE>;
  constexpr int ROW = ElemShape<NPE>::template pass_row<R>;
  constexpr int EPT = L::EPT;
  constexpr uint32_t STATE_BYTES = L::STATE_BYTES, NODE_BYTES = L::NODE_BYTES, IDX_BYTES = L::IDX_BYTES,
                     EMAT_BYTES = L::EMAT_BYTES, OFF_NODES = L::OFF_NODES, OFF_IDX = L::OFF_IDX,
                     IDX_STRIDE = L::IDX_STRIDE, OFF_CONN = L::OFF_CONN, OFF_ROWS = L::OFF_ROWS;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  auto state = [&](int b) { return reinterpret_cast<R *>(smem_raw + b * STATE_BYTES); };
  // node vector k (0 coordinates, 1 increments) of buffer b: xy then z arrays
  auto nxy = [&](int b, int k) {
    return reinterpret_cast<double2 *>(smem_raw + OFF_NODES + b * NODE_BYTES + k * TILE * (sizeof(double2) + sizeof(double)));
  };
  auto nz = [&](int b, int k) { return reinterpret_cast<double *>(nxy(b, k) + TILE); };
  auto spos = [&](int b) { return reinterpret_cast<int *>(smem_raw + OFF_IDX + b * IDX_STRIDE); };
  auto emat = [&](int b) { return reinterpret_cast<int *>(smem_raw + OFF_IDX + b * IDX_STRIDE + IDX_BYTES); };
  auto conn = [&](int c) { return reinterpret_cast<int *>(smem_raw + OFF_CONN + c * IDX_BYTES); };
  R *rows = reinterpret_cast<R *>(smem_raw + OFF_ROWS);
  __shared__ __align__(8) uint64_t sbar[2], cbar[3];
  const int t = threadIdx.x;
  const int lane = t & 31;
  const int g = lane & (NPE - 1);
  const int base = lane & ~(NPE - 1);
  if (t == 0)
  {
    mbar_init(&sbar[0], 1);
    mbar_init(&sbar[1], 1);
    mbar_init(&cbar[0], 1);
    mbar_init(&cbar[1], 1);
    mbar_init(&cbar[2], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto issue_state = [&](int tl, int b) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&sbar[b], STATE_BYTES + IDX_BYTES + EMAT_BYTES);
    bulk_g2s_ef(state(b), reinterpret_cast<const R *>(M.ip) + (size_t)tl * DNL_IP_NCOMP * TILE, STATE_BYTES, &sbar[b]);
    bulk_g2s(spos(b), M.slot_pos + (size_t)tl * TILE, IDX_BYTES, &sbar[b]);
    bulk_g2s(emat(b), M.emat + (size_t)tl * EPT, EMAT_BYTES, &sbar[b]);
  };
  auto issue_conn = [&](int tl, int c) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&cbar[c], IDX_BYTES);
    bulk_g2s(conn(c), M.conn + (size_t)tl * TILE, IDX_BYTES, &cbar[c]);
  };
  // this lane's node of a tile: coordinates and increment of field0 of the
  // slot's instance
  auto gather = [&](int inst, int c, int b) {
    const int node = conn(c)[t];
    const char *src_x = reinterpret_cast<const char *>(M.x + node);
    const char *src_u = reinterpret_cast<const char *>(M.u[M.ctl[inst].f0] + node);
    cp_async16(nxy(b, 0) + t, src_x);
    cp_async8(nz(b, 0) + t, src_x + 16);
    cp_async16(nxy(b, 1) + t, src_u);
    cp_async8(nz(b, 1) + t, src_u + 16);
    cp_async_commit();
  };
  uint32_t sph = 0, cph = 0; // parity bit of each barrier
  bool failed = false;
  auto wait_bar = [&](uint64_t *bar, uint32_t &bits, int k) {
    if (!failed && !mbar_wait(bar, (bits >> k) & 1u))
    {
      atomicExch(err, 1);
      failed = true;
    }
    bits ^= 1u << k;
  };

  // work slots (TileMap): this block's slots blockIdx.x, + gridDim.x, ...,
  // each a (tile, instance); cur, next and after are three consecutive ones
  const TileMap<NPE> map{M, nTiles};
  const int nSlots = map.count();
  struct Work
  {
    int slot, tile, inst;
  };
  auto work = [&](int slot) {
    Work w{slot, 0, 0};
    if (slot < nSlots)
      map.get(slot, w.tile, w.inst);
    return w;
  };
  Work cur = work(blockIdx.x);
  Work next = work(cur.slot + gridDim.x);
  if (t == 0 && cur.slot < nSlots)
  {
    issue_conn(cur.tile, 0);
    issue_state(cur.tile, 0);
    if (next.slot < nSlots)
      issue_conn(next.tile, 1);
  }
  if (cur.slot < nSlots)
  {
    wait_bar(&cbar[0], cph, 0);
    gather(cur.inst, 0, 0);
  }
  for (int b = 0, c = 0; cur.slot < nSlots; b ^= 1, c = (c == 2 ? 0 : c + 1))
  {
    const Work after = work(next.slot + gridDim.x);
    const int c1 = (c == 2 ? 0 : c + 1), c2 = (c1 == 2 ? 0 : c1 + 1);
    if (t == 0)
    {
      if (next.slot < nSlots)
        issue_state(next.tile, b ^ 1);
      if (after.slot < nSlots)
        issue_conn(after.tile, c2);
    }
    if (next.slot < nSlots)
    {
      wait_bar(&cbar[c1], cph, c1);
      gather(next.inst, c1, b ^ 1);
      cp_async_wait<1>(); // this tile's nodes (all but the group just issued)
    }
    else
      cp_async_wait<0>();
    wait_bar(&sbar[b], sph, b);
    const int q = cur.tile * TILE + t;
    const int e = q / NPE;
    Ctl *C = M.ctl + cur.inst;
    const bool act = e >= C->elem_begin && e < C->elem_end && C->active && !failed;
    const unsigned amask = __ballot_sync(0xffffffffu, act);
    if (act)
    {
      SharedTile<R> old{state(b), t};
      StagedIo<R, ONE> io{M, q, {nxy(b, 0) + t, nz(b, 0) + t}, {nxy(b, 1) + t, nz(b, 1) + t}, spos(b)[t],
                     M.mat + emat(b)[t / NPE], g};
      element_update<R, NPE>(io, C, q, e, g, base, amask, 0, old, rows + t * ROW, rows + (t - g) * ROW);
    }
    __syncthreads(); // the buffers of this tile are refilled from the next iteration on
    cur = next;
    next = after;
  }
  cp_async_wait<0>();
}

// ------------------------------------------------ element pass with modes

enum
{
  MODE_STATS = 1,   // Newton iterations counted
  MODE_HARVEST = 2, // + (trial state, converged gamma) pairs kept
  MODE_GUESS = 3    // + the network's guess as the first iterate
};

// Element pass (mixed precision) with the Newton iterations of the return
// counted, and, per MODE, training pairs harvested from the converged returns
// or the learned initial guess evaluated on the tensor cores for each tile of
// TILE points between the two halves of the update.  Persistent over tiles.
template <int NPE, int MODE>
__global__ void __launch_bounds__(TILE, 4) k_element_mode(DevModel M, int nTiles, int *err)
{
  using R = float;
  constexpr int ROW = ElemShape<NPE>::template pass_row<R>;
  __shared__ __align__(16) R sh[TILE * ROW];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tslot;
  extern __shared__ __align__(1024) unsigned char dyn[];
  const int t = threadIdx.x;
  const int lane = t & 31;
  const int g = lane & (NPE - 1);
  const int base = lane & ~(NPE - 1);
  mlp::Tile net;
  if constexpr (MODE == MODE_GUESS)
    mlp::tile_setup(net, dyn, M.mlp_image, &bar, &tslot, err);
  unsigned long long nEval = 0, nPlastic = 0, nScope = 0, nScopeEval = 0;
  for (int tile = blockIdx.x; tile < nTiles; tile += gridDim.x)
  {
    const int q = tile * TILE + t;
    const int e = q / NPE;
    const bool valid = e < M.nE;
    const int inst = (M.nInst > 1) ? find_segment(M.inst_elem_begin, M.nInst, valid ? e : M.nE - 1) : 0;
    Ctl *C = M.ctl + inst;
    const bool act = valid && C->active;
    const unsigned amask = __ballot_sync(0xffffffffu, act);
    R *row = sh + t * ROW, *grp = sh + (t - g) * ROW;
    GlobalState<R> old{M, q};
    EngineIo<R> io{M, q, act ? C->f0 : 0};
    Front<R> f;
    float x[mlp::NIN] = {0.f, 0.f, 0.f, 0.f, 0.f};
    float gmax = 0.f;
    bool plastic = false, scope = false;
    if (act)
    {
      element_front<R, NPE>(io, C, e, g, base, amask, M.conn[q], old, row, grp, f);
      const MatDev &mp = io.mat(e);
      JC<R> jc;
      jc.load(mp);
      const R dt = R(C->dt_eff), twoG = R(mp.twoG);
      R Strial, y0;
      trial_state<R>(jc, twoG, f.dE, f.st, dt, Strial, y0);
      plastic = Strial > y0;
      // first yield: no previous gamma to start from (Element.C:507-515)
      scope = plastic && (M.guess_scope == DNL_GUESS_ALL || f.st.epsp == R(0));
      if (plastic)
      {
        gmax = (Strial - y0) / (R(1.2247448713915890491) * twoG);
        mlp::features(Strial, f.st.epsp, f.st.depsp, f.st.T, twoG, dt, mp, x);
      }
    }
    R gamma0 = R(-1);
    if constexpr (MODE == MODE_GUESS)
    {
      __syncwarp();
      if (__syncthreads_or(scope))
      {
        const float y = net.forward(t, x);
        if (scope)
          gamma0 = fminf(fmaxf(mlp::ratio(net, y), 0.f), 2.f) * gmax;
      }
    }
    if (act)
    {
      const int evals = element_back<R, NPE>(io, C, q, e, g, amask, old, row, grp, f, gamma0);
      if (evals > 0)
      {
        nEval += evals;
        nPlastic++;
        if (scope)
        {
          nScopeEval += evals;
          nScope++;
        }
      }
      if constexpr (MODE == MODE_HARVEST)
      {
        const unsigned h = (unsigned)q * 2654435761u ^ (unsigned)C->inc * 40503u;
        if (scope && evals > 0 && gmax > 0.f && (h >> 7) % (unsigned)M.harvest_stride == 0u)
        {
          const unsigned long long k = atomicAdd(M.harvest_count, 1ull);
          if ((long long)k < M.harvest_cap)
          {
            float4 *o = reinterpret_cast<float4 *>(M.harvest + k * DNL_MLP_PAIR_WORDS);
            o[0] = make_float4(x[0], x[1], x[2], x[3]);
            o[1] = make_float4(x[4], f.st.gamma / gmax, f.st.gamma, gmax);
          }
        }
      }
    }
    __syncwarp();
  }
  // per-warp totals
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
  {
    nEval += __shfl_xor_sync(0xffffffffu, nEval, o);
    nPlastic += __shfl_xor_sync(0xffffffffu, nPlastic, o);
    nScope += __shfl_xor_sync(0xffffffffu, nScope, o);
    nScopeEval += __shfl_xor_sync(0xffffffffu, nScopeEval, o);
  }
  if (lane == 0 && nPlastic)
  {
    atomicAdd(M.stats + 0, nEval);
    atomicAdd(M.stats + 1, nPlastic);
    atomicAdd(M.stats + 2, nScope);
    atomicAdd(M.stats + 3, nScopeEval);
  }
  if constexpr (MODE == MODE_GUESS)
    mlp::tile_release(net);
}

// ------------------------------------------------------------ nodal update

// Explicit::computePredictions (Explicit.C:438-482) fused with
// Explicit::explicitSolve (Explicit.C:489-536): the nodal force is gathered
// from the element slots in element order (the order of the scatter-add of
// Model::computeInternalForces, Model.C:881-898), then the Chung-Hulbert
// corrector and the boundary conditions, then disp += du, coords += du.
//
// One thread per (node, component): the three components of the update are
// independent (the corrector, the boundary conditions and the nodal vectors
// all act component-wise), so a thread needs few registers and the pass runs
// at full occupancy, which is what hides the latency of its gather.  The
// component's force is still summed over the node's slots in element order.
constexpr int NODAL_THREADS = 128;
template <typename R, int DIM>
__device__ __forceinline__ void nodal_update(const DevModel &M, int i, int c, const Ctl *C)
{
  constexpr int BATCH = 8; // slots loaded together
  constexpr int W = DIM == 3 ? 8 : 4; // the fixed-stride layout's slots per node
  const double m = M.mass[i];
  const unsigned code = (M.bc[i] >> (2 * c)) & 3u;
  const double X = reinterpret_cast<const double *>(M.x + i)[c];
  const double D = reinterpret_cast<const double *>(M.disp + i)[c];
  if (!C->active)
    return;
  const int f0 = C->f0, f1 = 1 - f0;
  double v0 = reinterpret_cast<const double *>(M.v[f0] + i)[c];
  double a0 = reinterpret_cast<const double *>(M.a[f0] + i)[c];
  // this component of the node's slots (4 values per slot), summed in element order
  const R *sc = reinterpret_cast<const R *>(M.slot) + c;
  double f = 0.0;
  if (M.slotW == W)
  {
    // fixed stride: no offsets to load first; the padding adds zeros
    R s[W];
#pragma unroll
    for (int j = 0; j < W; j++)
      s[j] = sc[4 * (W * i + j)];
#pragma unroll
    for (int j = 0; j < W; j++)
      f += (double)s[j];
  }
  else
  {
    const int kb = M.csr_off[i], ke = M.csr_off[i + 1];
    for (int k0 = kb; k0 < ke; k0 += BATCH)
    {
      R s[BATCH];
#pragma unroll
      for (int j = 0; j < BATCH; j++)
        if (k0 + j < ke)
          s[j] = sc[4 * (k0 + j)];
#pragma unroll
      for (int j = 0; j < BATCH; j++)
        if (k0 + j < ke)
          f += (double)s[j];
    }
  }
  const double dt = C->dt_eff, t = C->t;
  const double beta = C->beta, gam = C->gammaN, alphaM = C->alphaM;
  double du = dt * (v0 + (0.5 - beta) * dt * a0);
  double v1 = v0 + (1.0 - gam) * dt * a0;
  double a1 = (c < DIM) ? f / m : 0.0;
  a1 = (a1 - alphaM * a0) / (1.0 - alphaM);
  v1 += gam * dt * a1;
  du += beta * (dt * dt) * a1;
  // the z thread also writes the (zero) fourth word, so that every 32-byte
  // sector of the node vectors is written whole (a partly written sector
  // costs a read of it from DRAM when it leaves the L2)
  auto put = [&](double4 *v, double val) {
    if (c == 2)
      reinterpret_cast<double2 *>(v)[1] = make_double2(val, 0.0);
    else
      reinterpret_cast<double *>(v)[c] = val;
  };
  if (code == DNL_BC_RESTRAIN)
  {
    // BoundaryRestrain.C:98-128 (both fields)
    du = v1 = a1 = 0.0;
    put(M.u[f0] + i, 0.0);
    put(M.v[f0] + i, 0.0);
    put(M.a[f0] + i, 0.0);
  }
  else if (code == DNL_BC_SPEED)
  {
    // BoundarySpeed.C:139-206 (both fields)
    const double sv = reinterpret_cast<const double *>(M.bcval + i)[c];
    const int fn = reinterpret_cast<const int *>(M.bcfun + i)[c];
    double va = sv, vb = sv, acc = 0.0;
    if (fn >= 0)
    {
      const double fa = func_value(M, fn, t), fb = func_value(M, fn, t + dt);
      acc = (fb - fa) * sv / dt;
      va = fa * sv;
      vb = fb * sv;
    }
    a1 = acc;
    v1 = vb;
    du = vb * dt;
    put(M.u[f0] + i, va * dt);
    put(M.v[f0] + i, va);
    put(M.a[f0] + i, acc);
  }
  put(M.x + i, X + du);
  put(M.disp + i, D + du);
  put(M.u[f1] + i, du);
  put(M.v[f1] + i, v1);
  put(M.a[f1] + i, a1);
}

// A single model: one thread per (node, component).
template <typename R, int DIM>
__global__ void __launch_bounds__(NODAL_THREADS) k_nodal(DevModel M)
{
  pdl_wait();
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k == 0) // for the Courant pass that follows (k_courant_finish)
    *M.step_due = M.ctl[0].active && M.ctl[0].due;
  const int i = (int)(k / 3), c = (int)(k - 3LL * i);
  if (i < M.nN)
    nodal_update<R, DIM>(M, i, c, M.ctl);
}

// A batch: a grid-stride loop over the (node, component) pairs of the running
// instances only (k_active_list), so that stopped instances cost nothing.
template <typename R, int DIM>
__global__ void __launch_bounds__(NODAL_THREADS) k_nodal_batch(DevModel M)
{
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k == 0)
    *M.step_due = 1u;
  const int na = *M.act_count;
  const long long n3 = 3LL * M.act_node_pre[na];
  for (long long kk = k; kk < n3; kk += (long long)gridDim.x * blockDim.x)
  {
    const int j = (int)(kk / 3), c = (int)(kk - 3LL * j);
    const int a = find_segment(M.act_node_pre, na, j);
    const Ctl *C = M.ctl + M.act_list[a];
    nodal_update<R, DIM>(M, C->node_begin + (j - M.act_node_pre[a]), c, C);
  }
}

// Predictor boundary conditions on field0 of the imposed-speed nodes before the
// element pass (the element pass reads field0->u, Element.C:1114).
__global__ void k_bc_prep(DevModel M)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= M.nSpeed)
    return;
  const int i = M.speed_nodes[k];
  const int inst = (M.nInst > 1) ? find_segment(M.inst_node_begin, M.nInst, i) : 0;
  const Ctl *C = M.ctl + inst;
  if (!C->active)
    return;
  const double dt = C->dt_eff, t = C->t;
  const int f0 = C->f0;
  const unsigned code = M.bc[i];
  double4 u0 = M.u[f0][i], v0 = M.v[f0][i], a0 = M.a[f0][i];
  const double4 sv = M.bcval[i];
  const int4 sf = M.bcfun[i];
  for (int c = 0; c < 3; c++)
  {
    if (((code >> (2 * c)) & 3u) != DNL_BC_SPEED)
      continue;
    double4 svc = sv;
    const double s = comp(svc, c);
    const int fn = c == 0 ? sf.x : (c == 1 ? sf.y : sf.z);
    double va = s, acc = 0.0;
    if (fn >= 0)
    {
      const double fa = func_value(M, fn, t), fb = func_value(M, fn, t + dt);
      acc = (fb - fa) * s / dt;
      va = fa * s;
    }
    comp(a0, c) = acc;
    comp(v0, c) = va;
    comp(u0, c) = va * dt;
  }
  M.u[f0][i] = u0;
  M.v[f0][i] = v0;
  M.a[f0][i] = a0;
}

// Sum the element slots of every node (lumped mass at the start, or the
// internal forces for the kernel-level entry point).
template <typename R>
__global__ void k_gather(DevModel M, int what)
{
  using R4 = typename V4<R>::type;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M.nN)
    return;
  const R4 *slot = reinterpret_cast<const R4 *>(M.slot);
  double4 f = make_double4(0, 0, 0, 0);
  const int kb = slot_begin(M, i), ke = kb + M.csr_off[i + 1] - M.csr_off[i];
  for (int k = kb; k < ke; k++)
  {
    const R4 s = slot[k];
    f.x += (double)s.x;
    f.y += (double)s.y;
    f.z += (double)s.z;
  }
  if (what == 0)
    M.mass[i] = f.x;
  else
    M.fout[i] = f;
}

// ---------------------------------------------------------------- control

enum
{
  CTL_FINISH = 0,   // end of the increment that ran, then begin the next one
  CTL_LIMITS = 1,   // new pause time / increment budget, then begin
  CTL_INIT_DT = 2,  // after the forced Courant pass of the start: dt, then arm the first element pass
  CTL_POST_INIT = 3 // after the first element pass
};

__device__ __forceinline__ void begin_increment(Ctl &c)
{
  // Explicit::updateTimes (Explicit.C:414-427) for the increment to come
  const bool go = c.status == 0 && c.t < c.t_end && c.t < c.t_stop && c.inc < c.inc_stop;
  if (go)
  {
    if (c.t + c.dt > c.t_end)
      c.dt = c.t_end - c.t;
    c.inc += 1;
    c.dt_eff = c.dt;
    c.t_new = c.t + c.dt;
    // Solver::computeTimeStep runs after the Jacobian when the solve goes on (Explicit.C:239-254, Solver.C:200)
    c.due = (c.t_new < c.t_end) && (c.inc % c.ts_freq == 0);
  }
  else
    c.due = 0;
  c.active = go;
  c.prepared = 1;
}

__device__ __forceinline__ void apply_courant(Ctl &c)
{
  // Solver::computeTimeStep (Solver.C:205-226): omega_max = 2 / dt_crit, or
  // the power-iteration omega_max (Model.C:1008)
  if (c.ts_method == DNL_TS_POWER_ITERATION)
    c.dt = c.safety * c.omegaS / c.pi_omega;
  else
  {
    const double crit = __longlong_as_double((long long)c.min_bits);
    c.dt = c.safety * c.omegaS / (2.0 / crit);
  }
  c.min_bits = INF_BITS;
}

// end of the increment that ran, then begin the next one
__device__ __forceinline__ void finish_increment(Ctl &c)
{
  if (c.prepared && c.active && c.status == 0)
  {
    // Explicit::endStep (Explicit.C:539-552): time, then the nodal field swap
    c.t = c.t_new;
    c.dt_last = c.dt_eff;
    c.f0 ^= 1;
    if (c.due)
      apply_courant(c);
  }
  c.prepared = 0;
  c.active = 0;
  begin_increment(c);
}

__global__ void k_control(DevModel M, int phase, double t_stop, long long max_incs)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M.nInst)
    return;
  Ctl &c = M.ctl[i];
  if (phase == CTL_FINISH)
    finish_increment(c);
  else if (phase == CTL_LIMITS)
  {
    const long long committed = c.inc - ((c.prepared && c.active) ? 1 : 0);
    c.inc = committed;
    c.t_stop = t_stop;
    c.inc_stop = (max_incs > 0) ? committed + max_incs : 0x7fffffffffffffffll;
    c.prepared = 0;
    c.active = 0;
    begin_increment(c);
  }
  else if (phase == CTL_INIT_DT)
  {
    apply_courant(c);
    c.dt_eff = c.dt;
    c.active = (c.status == 0);
    c.prepared = 0;
    c.due = 0;
  }
  else
  {
    c.active = 0;
    c.prepared = 0;
  }
}

// ------------------------------------------------------------- time step

__device__ __forceinline__ double3 d3(const double4 &v) { return make_double3(v.x, v.y, v.z); }
__device__ __forceinline__ double3 sub(double3 a, double3 b) { return make_double3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ double3 cross(double3 a, double3 b)
{
  return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double norm(double3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ double dot(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// ElHex8N3D::getCharacteristicLength (ElHex8N3D.C:634-649): volume
// (ElHex8N3D::getVolume, three pyramids with apex at node 7, ElHex8N3D.C:651-686)
// over the largest face area (half the cross product of the face diagonals).
__device__ __forceinline__ double charlen_hex(const double3 P[8])
{
  const int faces[6][4] = {{0, 1, 2, 3}, {0, 1, 5, 4}, {1, 2, 6, 5}, {3, 2, 6, 7}, {0, 3, 7, 4}, {4, 5, 6, 7}};
  double amax = 0.0;
#pragma unroll
  for (int f = 0; f < 6; f++)
  {
    const double a = 0.5 * norm(cross(sub(P[faces[f][0]], P[faces[f][2]]), sub(P[faces[f][1]], P[faces[f][3]])));
    amax = fmax(amax, a);
  }
  double vol = 0.0;
#pragma unroll
  for (int k = 0; k < 3; k++)
  {
    const double3 A = P[faces[k][0]], B = P[faces[k][1]], Cc = P[faces[k][2]], D = P[faces[k][3]];
    const double3 ab = sub(B, A), ac = sub(Cc, A), ad = sub(D, A);
    const double area = (norm(cross(ab, ac)) + norm(cross(ad, ac))) / 2.0;
    double3 nr = cross(ab, ad);
    const double nn = norm(nr);
    nr = make_double3(nr.x / nn, nr.y / nn, nr.z / nn);
    const double h = fabs(dot(nr, sub(P[7], A)));
    vol += area * h / 3.0;
  }
  return vol / amax;
}

// ElQua4NAx::getCharacteristicLength (ElQua4NAx.C:312-321).
__device__ __forceinline__ double charlen_q4(const double3 P[4])
{
  const double x31 = P[2].x - P[0].x, x24 = P[1].x - P[3].x, y42 = P[3].y - P[1].y, y31 = P[2].y - P[0].y;
  return (x31 * y42 + x24 * y31) / sqrt(2.0 * (x24 * x24 + y42 * y42 + x31 * x31 + y31 * y31));
}

// Model::computeCourantTimeStep (Model.C:636-669): min over elements of l_e/c_e
// with the elongation wave speed of the mean point density (Element.C:343-359).
// One thread per element, a segmented warp-shuffle min over the lanes of one
// instance, then one atomicMin per instance and warp (called by a full warp).
template <typename R, int NPE>
__device__ __forceinline__ void courant_warp(const DevModel &M, int e, int lane, int inst, bool act, Ctl *C)
{
  double ratio = 1e300;
  if (act)
  {
    double3 P[NPE];
#pragma unroll
    for (int n = 0; n < NPE; n++)
      P[n] = d3(M.x[M.conn[e * NPE + n]]);
    double len;
    if constexpr (NPE == 8)
      len = charlen_hex(P);
    else
      len = charlen_q4(P);
    double rho = 0.0;
#pragma unroll
    for (int g = 0; g < NPE; g++)
      rho += (double)ipv<R>(M, DNL_IP_DENSITY, e * NPE + g);
    rho /= NPE;
    const MatDev &mp = M.mat[M.emat[e]];
    ratio = len / sqrt(mp.wave2 / rho);
  }
  // segmented min: lanes of one instance form a contiguous run
  const int key = act ? inst : -1;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1)
  {
    const double o = __shfl_down_sync(0xffffffffu, ratio, off);
    const int ok = __shfl_down_sync(0xffffffffu, key, off);
    if (lane + off < 32 && ok == key)
      ratio = fmin(ratio, o);
  }
  const int prev = __shfl_up_sync(0xffffffffu, key, 1);
  if (act && (lane == 0 || prev != key))
    atomicMin(&C->min_bits, (unsigned long long)__double_as_longlong(ratio));
}

template <typename R, int NPE>
__global__ void __launch_bounds__(256) k_courant(DevModel M, int force)
{
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool valid = e < M.nE;
  const int ec = valid ? e : M.nE - 1;
  const int inst = (M.nInst > 1) ? find_segment(M.inst_elem_begin, M.nInst, ec) : 0;
  Ctl *C = M.ctl + inst;
  const bool act = valid && (force || (C->active && C->due));
  if (__ballot_sync(0xffffffffu, act) == 0)
    return;
  courant_warp<R, NPE>(M, e, lane, inst, act, C);
}

// The Courant pass of an increment fused with the end of the increment:
// persistent over elements (it only works every ts_freq increments), and the
// block that finishes last runs finish_increment for every instance (what
// k_control(CTL_FINISH) does), one launch instead of two.
template <typename R, int NPE>
__global__ void __launch_bounds__(256) k_courant_finish(DevModel M)
{
  pdl_wait();
  const int lane = threadIdx.x & 31;
  const int stride = gridDim.x * blockDim.x;
  const int nE32 = (M.nE + 31) & ~31; // whole warps, so every lane takes the same trips
  // read from the flag the nodal pass wrote, not from the control block, which
  // the block that finishes the increment rewrites while others may still read
  if (*M.step_due == 0u)
  {
    // a single model whose time step is not due: no minimum to wait for, the
    // first block finishes the increment and the others leave at once
    if (blockIdx.x == 0 && threadIdx.x == 0)
      finish_increment(M.ctl[0]);
    return;
  }
  if (M.nInst == 1)
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nE32; e += stride)
    {
      const bool valid = e < M.nE;
      Ctl *C = M.ctl;
      const bool act = valid && C->active && C->due;
      if (__ballot_sync(0xffffffffu, act) != 0)
        courant_warp<R, NPE>(M, valid ? e : M.nE - 1, lane, 0, act, C);
    }
  else
  {
    // the elements of the running instances whose time step is due (k_active_list)
    const int na = *M.due_count;
    const int nAct = M.due_elem_pre[na], nAct32 = (nAct + 31) & ~31;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nAct32; k += stride)
    {
      const bool valid = k < nAct;
      const int kc = valid ? k : nAct - 1;
      const int a = find_segment(M.due_elem_pre, na, kc);
      const int inst = M.due_list[a];
      Ctl *C = M.ctl + inst;
      const int e = C->elem_begin + (kc - M.due_elem_pre[a]);
      const bool act = valid && C->active && C->due;
      if (__ballot_sync(0xffffffffu, act) != 0)
        courant_warp<R, NPE>(M, e, lane, inst, act, C);
    }
  }
  // last block done: every block's minima are in memory before it counts itself
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0)
    last = atomicAdd(M.done_count, 1u) == gridDim.x - 1;
  __syncthreads();
  if (last)
  {
    __threadfence();
    for (int i = threadIdx.x; i < M.nInst; i += blockDim.x)
      finish_increment(M.ctl[i]);
    if (threadIdx.x == 0)
      *M.done_count = 0;
  }
}

// ------------------------------------------------- power-iteration time step

// K_e v_e of one element at this lane's Gauss point, added over the element's
// points through shared memory (ElementPlane.C:182-292, Element3D.C:303-399,
// applied without forming K_e): eps = B v (Voigt, engineering shear), sig = C eps
// with the Hooke matrices of Material.C:98-152 (shear modulus term E/(1+nu)),
// y_n = B_n^T sig w detJ (x 2 pi r, + the hoop row for axisymmetric elements).
template <int NPE>
__device__ __forceinline__ void element_Kv(const DevModel &M, int q, int e, int g, int base, unsigned amask,
                                           const double *v, double scale, double *row, double *grp)
{
  constexpr int DIM = ElemShape<NPE>::DIM;
  const bool AXI = ElemShape<NPE>::AXI && !M.ctl[0].plane;
  constexpr int ROW = ElemShape<NPE>::ROW;
  const int node = M.conn[q];
  const MatDev &mp = M.mat[M.emat[e]];
  double detJ, inv[3][3], radius, H[9];
  const double4 Xn = M.x[node], Un = make_double4(0, 0, 0, 0);
  double4 X0, U0;
  first_node_by_shuffle(amask, base, Xn, Un, X0, U0);
  kinematics<double, NPE>(amask, g, base, Xn, Un, X0, U0, detJ, inv, radius, H, AXI, (double *)nullptr);
  double WxdJ = detJ;
  if (AXI)
    WxdJ *= 6.28318530717958647692 * radius;
  const double vx = v[3 * node] * scale, vy = v[3 * node + 1] * scale, vz = DIM == 3 ? v[3 * node + 2] * scale : 0.0;
  const double a = 0.57735026918962576451;
  const double xi0 = node_sign(g, 0) * a, xi1 = node_sign(g, 1) * a, xi2 = node_sign(g, 2) * a;
  // strains of B v
  double eps[6] = {0, 0, 0, 0, 0, 0};
  double dNx[NPE][3], Nv[NPE];
#pragma unroll
  for (int n = 0; n < NPE; n++)
  {
    double dxi[3], Nn;
    switch (n)
    {
#define DNL_SHAPE_CASE(K)                                                                                          \
  case K:                                                                                                          \
    shape<double, NPE, (K < NPE ? K : 0)>(xi0, xi1, xi2, dxi, Nn);                                                  \
    break;
      DNL_SHAPE_CASE(0) DNL_SHAPE_CASE(1) DNL_SHAPE_CASE(2) DNL_SHAPE_CASE(3) DNL_SHAPE_CASE(4) DNL_SHAPE_CASE(5)
      DNL_SHAPE_CASE(6) DNL_SHAPE_CASE(7)
#undef DNL_SHAPE_CASE
    }
#pragma unroll
    for (int k = 0; k < 3; k++)
    {
      double s_ = 0.0;
#pragma unroll
      for (int j = 0; j < DIM; j++)
        s_ += dxi[j] * inv[j][k];
      dNx[n][k] = (k < DIM) ? s_ : 0.0;
    }
    Nv[n] = Nn;
    const double ux = __shfl_sync(amask, vx, base + n), uy = __shfl_sync(amask, vy, base + n),
                 uz = DIM == 3 ? __shfl_sync(amask, vz, base + n) : 0.0;
    if constexpr (DIM == 3)
    {
      eps[0] += dNx[n][0] * ux;
      eps[1] += dNx[n][1] * uy;
      eps[2] += dNx[n][2] * uz;
      eps[3] += dNx[n][1] * ux + dNx[n][0] * uy;
      eps[4] += dNx[n][2] * uy + dNx[n][1] * uz;
      eps[5] += dNx[n][2] * ux + dNx[n][0] * uz;
    }
    else
    {
      eps[0] += dNx[n][0] * ux;
      eps[1] += dNx[n][1] * uy;
      eps[2] += dNx[n][1] * ux + dNx[n][0] * uy;
      if (AXI)
        eps[3] += Nn / radius * ux;
    }
  }
  const double E = mp.young, nu = mp.poisson, f = E / ((1 + nu) * (1 - 2 * nu));
  const double cd = (1 - nu) * f, co = nu * f, cs = (1 - 2 * nu) * f;
  double sig[6];
  if constexpr (DIM == 3)
  {
    sig[0] = cd * eps[0] + co * (eps[1] + eps[2]);
    sig[1] = cd * eps[1] + co * (eps[0] + eps[2]);
    sig[2] = cd * eps[2] + co * (eps[0] + eps[1]);
    sig[3] = cs * eps[3];
    sig[4] = cs * eps[4];
    sig[5] = cs * eps[5];
  }
  else
  {
    sig[0] = cd * eps[0] + co * (eps[1] + eps[3]);
    sig[1] = cd * eps[1] + co * (eps[0] + eps[3]);
    sig[2] = cs * eps[2];
    sig[3] = cd * eps[3] + co * (eps[0] + eps[1]);
  }
#pragma unroll
  for (int n = 0; n < NPE; n++)
  {
    if constexpr (DIM == 3)
    {
      row[n * 3] = (dNx[n][0] * sig[0] + dNx[n][1] * sig[3] + dNx[n][2] * sig[5]) * WxdJ;
      row[n * 3 + 1] = (dNx[n][1] * sig[1] + dNx[n][0] * sig[3] + dNx[n][2] * sig[4]) * WxdJ;
      row[n * 3 + 2] = (dNx[n][2] * sig[2] + dNx[n][1] * sig[4] + dNx[n][0] * sig[5]) * WxdJ;
    }
    else
    {
      row[n * 2] = (dNx[n][0] * sig[0] + dNx[n][1] * sig[2] + (AXI ? Nv[n] / radius * sig[3] : 0.0)) * WxdJ;
      row[n * 2 + 1] = (dNx[n][1] * sig[1] + dNx[n][0] * sig[2]) * WxdJ;
    }
  }
  __syncwarp(amask);
  double4 y = make_double4(0, 0, 0, 0);
#pragma unroll
  for (int l = 0; l < NPE; l++)
  {
    y.x += grp[l * ROW + g * DIM];
    y.y += grp[l * ROW + g * DIM + 1];
    if constexpr (DIM == 3)
      y.z += grp[l * ROW + g * DIM + 2];
  }
  M.pislot[M.slot_pos[q]] = y;
}

// Model::computePowerIterationTimeStep (Model.C:942-1009) for a single model,
// as one cooperative kernel: each iteration is an element phase (K v into the
// slots), a grid barrier, a node phase (v_new = (v + sum of the node's slots in
// element order) / m, block maxima of |v_new|), a grid barrier and the
// convergence test |fmax - fmax_prev| / fmax < 1e-4, at most 1000 iterations.
// v is kept unnormalised between iterations (scale = 1 / fmax).  Runs only
// when the time step is due (or forced at the start).
template <int NPE>
__global__ void __launch_bounds__(TILE) k_power_iteration(DevModel M, int force)
{
  constexpr int ROW = ElemShape<NPE>::ROW;
  constexpr int DIM = ElemShape<NPE>::DIM;
  __shared__ double sh[TILE * ROW];
  __shared__ double red[TILE / 32];
  Ctl *C = M.ctl;
  if (!(force || (C->active && C->due)))
    return;
  cooperative_groups::grid_group grid = cooperative_groups::this_grid();
  const int t = threadIdx.x, lane = t & 31;
  const int g = lane & (NPE - 1), base = lane & ~(NPE - 1);
  const int nTiles = (M.nE * NPE + TILE - 1) / TILE;
  double *v = M.pv, *vn = M.pv2;
  double scale = 1.0, fprev = C->pi_fmax, fmx = 0.0;
  int it = 0;
  bool ok = false;
  while (!ok)
  {
    it++;
    for (int tile = blockIdx.x; tile < nTiles; tile += gridDim.x)
    {
      const int q = tile * TILE + t, e = q / NPE;
      const bool act = e < M.nE;
      const unsigned amask = __ballot_sync(0xffffffffu, act);
      if (act)
        element_Kv<NPE>(M, q, e, g, base, amask, v, scale, sh + t * ROW, sh + (t - g) * ROW);
      __syncwarp();
    }
    grid.sync();
    double lmax = 0.0;
    for (int i = blockIdx.x * blockDim.x + t; i < M.nN; i += gridDim.x * blockDim.x)
    {
      double acc[3] = {v[3 * i] * scale, v[3 * i + 1] * scale, v[3 * i + 2] * scale};
      const int kb = slot_begin(M, i), ke = kb + M.csr_off[i + 1] - M.csr_off[i];
      for (int k = kb; k < ke; k++)
      {
        const double4 y = M.pislot[k];
        acc[0] += y.x;
        acc[1] += y.y;
        acc[2] += y.z;
      }
      const double m = M.mass[i];
#pragma unroll
      for (int c = 0; c < 3; c++)
      {
        const double val = (c < DIM) ? acc[c] / m : 0.0;
        vn[3 * i + c] = val;
        lmax = fmax(lmax, fabs(val));
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
      lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, off));
    if (lane == 0)
      red[t / 32] = lmax;
    __syncthreads();
    if (t == 0)
    {
      double b = 0.0;
      for (int w = 0; w < TILE / 32; w++)
        b = fmax(b, red[w]);
      M.blockmax[blockIdx.x] = b;
    }
    grid.sync();
    fmx = 0.0;
    for (int b = 0; b < (int)gridDim.x; b++)
      fmx = fmax(fmx, M.blockmax[b]);
    ok = fabs(fmx - fprev) / fmx < 1e-4;
    fprev = fmx;
    scale = 1.0 / fmx;
    double *tmp = v;
    v = vn;
    vn = tmp;
    if (it > 1000 && !ok)
    {
      if (blockIdx.x == 0 && t == 0)
        raise_status(C, DNL_ERR_POWER_ITERATION, it);
      return;
    }
  }
  // keep the normalised vector and the frequency for the next call (warm start)
  for (int i = blockIdx.x * blockDim.x + t; i < 3 * M.nN; i += gridDim.x * blockDim.x)
    M.pv[i] = v[i] * scale;
  if (blockIdx.x == 0 && t == 0)
  {
    C->pi_fmax = fmx;
    C->pi_omega = sqrt(fmx);
    C->pi_iters += it;
  }
}

// ------------------------------------------------------------ model build
//
// The model is built on the device from the caller's arrays as they come
// (uploaded into scratch): node vectors in the double4 layout, boundary codes,
// connectivity with each instance's node offset, element materials, and the
// node -> slot lists (CSR) of the force assembly.

// Per instance: first node, first element, first material, first function.
struct BuildRaw
{
  const double *coords, *vinit, *bcval; // [3 nN]
  const int8_t *bccode;                 // [3 nN]
  const int *bcfun;                     // [3 nN], -1 none
  const int *conn;                      // [nIP], instance-local node indices
  const int *emat;                      // [nE], instance-local material indices
  const int4 *base;                     // [nInst]: node, element, material, function bases
  int *speedCount;                      // nodes with an imposed speed (list fill)
  int *cursor;                          // [nN] CSR fill cursors
  int *list;                            // [nIP] incidences grouped by node
  int *blockSums;                       // scan partials
  int *maxValence;                      // largest slot count of a node
  const int *ext_of;                    // [nN] the caller's node of each engine node, or nullptr
  const int *int_of;                    // [nN] the engine's node of each caller's node, or nullptr
  int npe;
};

// Nodes: coordinates, initial speed (the description's, then the imposed
// speed of a constant condition, Model.C:429 / BoundarySpeed.C:63-73), zero
// displacement, increments and accelerations, boundary codes (an imposed zero
// speed restrains the component), imposed speeds and their functions.
__global__ void k_build_nodes(DevModel M, BuildRaw R, int hasSpeed)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M.nN)
    return;
  const int inst = (M.nInst > 1) ? find_segment(M.inst_node_begin, M.nInst, i) : 0;
  const int fbase = R.base[inst].w;
  const double4 zero = make_double4(0, 0, 0, 0);
  const int r = R.ext_of ? R.ext_of[i] : i; // where the caller's arrays hold this node
  double4 v = make_double4(R.vinit[3 * r], R.vinit[3 * r + 1], R.vinit[3 * r + 2], 0.0);
  double4 sv = zero;
  int4 sf = make_int4(-1, -1, -1, -1);
  unsigned code = 0;
  bool speed = false;
  for (int c = 0; c < 3; c++)
  {
    int cc = R.bccode[3 * r + c];
    const double val = R.bcval[3 * r + c];
    const int fn = R.bcfun[3 * r + c];
    if (cc == DNL_BC_SPEED && val == 0.0)
      cc = DNL_BC_RESTRAIN;
    if (cc == DNL_BC_SPEED)
    {
      speed = true;
      comp(sv, c) = val;
      (c == 0 ? sf.x : (c == 1 ? sf.y : sf.z)) = fn >= 0 ? fn + fbase : -1;
    }
    if (cc == DNL_BC_RESTRAIN || cc == DNL_BC_SPEED)
      code |= (unsigned)cc << (2 * c);
  }
  if (speed)
  {
    v = sv;
    const_cast<int *>(M.speed_nodes)[atomicAdd(R.speedCount, 1)] = i;
  }
  M.x[i] = make_double4(R.coords[3 * r], R.coords[3 * r + 1], R.coords[3 * r + 2], 0.0);
  M.v[0][i] = v;
  M.v[1][i] = v;
  M.disp[i] = zero;
  M.u[0][i] = M.u[1][i] = zero;
  M.a[0][i] = M.a[1][i] = zero;
  const_cast<uint8_t *>(M.bc)[i] = (uint8_t)code;
  if (hasSpeed)
  {
    const_cast<double4 *>(M.bcval)[i] = sv;
    const_cast<int4 *>(M.bcfun)[i] = sf;
  }
}

// Connectivity (with the instance's node offset; whole tiles, the padding
// zero), element materials, and each node's slot count in csr_off[node + 1].
__global__ void k_build_elems(DevModel M, BuildRaw R, int nIPpad)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nIPpad)
    return;
  int *conn = const_cast<int *>(M.conn);
  int *off = const_cast<int *>(M.csr_off);
  int *emat = const_cast<int *>(M.emat);
  const int e = k / R.npe;
  if (k >= M.nIP)
  {
    conn[k] = 0;
    const_cast<int *>(M.slot_pos)[k] = 0;
    if (k % R.npe == 0)
      emat[e] = 0;
    return;
  }
  const int inst = (M.nInst > 1) ? find_segment(M.inst_elem_begin, M.nInst, e) : 0;
  const int4 b = R.base[inst];
  const int node = R.int_of ? R.int_of[R.conn[k] + b.x] : R.conn[k] + b.x;
  conn[k] = node;
  atomicAdd(&off[node + 1], 1);
  if (k % R.npe == 0)
    emat[e] = b.z + R.emat[e];
}

// Inclusive scan of csr_off[1 .. nN] in three launches: per-block scans with
// their totals, a scan of the totals (one block), the totals added back.
constexpr int SCAN_BLOCK = 1024;
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_blocks(int *a, int n, int *blockSums)
{
  __shared__ int wsum[32];
  const int i = blockIdx.x * SCAN_BLOCK + threadIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int v = i < n ? a[i] : 0;
  for (int o = 1; o < 32; o <<= 1)
  {
    const int y = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o)
      v += y;
  }
  if (lane == 31)
    wsum[w] = v;
  __syncthreads();
  if (w == 0)
  {
    int x = wsum[lane];
    for (int o = 1; o < 32; o <<= 1)
    {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o)
        x += y;
    }
    wsum[lane] = x;
  }
  __syncthreads();
  if (w > 0)
    v += wsum[w - 1];
  if (i < n)
    a[i] = v;
  if (threadIdx.x == SCAN_BLOCK - 1)
    blockSums[blockIdx.x] = v;
}
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_sums(int *blockSums, int nb)
{
  if (threadIdx.x == 0)
  {
    int run = 0;
    for (int b = 0; b < nb; b++)
    {
      run += blockSums[b];
      blockSums[b] = run;
    }
  }
}
__global__ void k_scan_add(int *a, int n, const int *blockSums)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && i >= SCAN_BLOCK)
    a[i] += blockSums[i / SCAN_BLOCK - 1];
}

// Slot lists: each incidence appended to its node's run (any order), then
// each run sorted by incidence (the element order of the reference's
// scatter-add, Model.C:881-898) and slot_pos[k] set to k's place.
__global__ void k_slot_cursor(DevModel M, BuildRaw R)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < M.nN)
    R.cursor[i] = M.csr_off[i];
}
__global__ void k_slot_fill(DevModel M, BuildRaw R)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < M.nIP)
    R.list[atomicAdd(&R.cursor[M.conn[k]], 1)] = k;
}
__global__ void k_slot_sort(DevModel M, BuildRaw R)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M.nN)
    return;
  const int b = M.csr_off[i], n = M.csr_off[i + 1] - b;
  int *L = R.list + b;
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
  atomicMax(R.maxValence, n);
}
// slot_pos in the fixed-stride layout of W slots per node when no node has
// more (the host reads the same decision back), else in the CSR layout
__global__ void k_slot_pos(DevModel M, BuildRaw R, int W)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M.nN)
    return;
  const int b = M.csr_off[i], n = M.csr_off[i + 1] - b;
  const int first = (*R.maxValence <= W) ? W * i : b;
  const int *L = R.list + b;
  int *pos = const_cast<int *>(M.slot_pos);
  for (int j = 0; j < n; j++)
    pos[L[j]] = first + j;
}

// ------------------------------------------------------- state read-back

// Nodal vector `field` (DNL_NODE_*) of node i, on the parity of the two-buffer
// fields of the node's instance (field0 = the current values; the _PREV
// fields the other buffer, the values before the last increment).
__device__ __forceinline__ double4 node_vec(const DevModel &M, int field, int i)
{
  const int inst = (M.nInst > 1) ? find_segment(M.inst_node_begin, M.nInst, i) : 0;
  const int f0 = M.ctl[inst].f0;
  double4 v = make_double4(0, 0, 0, 0);
  switch (field)
  {
  case DNL_NODE_COORDS: v = M.x[i]; break;
  case DNL_NODE_DISP: v = M.disp[i]; break;
  case DNL_NODE_U: v = M.u[f0][i]; break;
  case DNL_NODE_SPEED: v = M.v[f0][i]; break;
  case DNL_NODE_ACCEL: v = M.a[f0][i]; break;
  case DNL_NODE_SPEED_PREV: v = M.v[1 - f0][i]; break;
  case DNL_NODE_U_PREV: v = M.u[1 - f0][i]; break;
  case DNL_NODE_ACCEL_PREV: v = M.a[1 - f0][i]; break;
  case DNL_NODE_FORCE: v = M.fout[i]; break;
  case DNL_NODE_MASS: v.x = v.y = v.z = M.mass[i]; break;
  default: break;
  }
  return v;
}

// Nodal vector `field` of nodes [n0, n0 + n) as [n][3] FP64 (the layout of
// dnl_engine_get_nodes), packed on the device so that one copy brings it out.
// perm: the engine's node of each caller's node, or nullptr (same numbering)
__global__ void k_nodes_out(DevModel M, int field, int n0, int n, double *dst, const int *perm)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n)
    return;
  const double4 v = node_vec(M, field, perm ? perm[n0 + k] : n0 + k);
  dst[3 * k] = v.x;
  dst[3 * k + 1] = v.y;
  dst[3 * k + 2] = v.z;
}

// Incidence (e * npe + local node) of each force slot: the inverse of slot_pos.
__global__ void k_slot_incidence(DevModel M, int *slot_inc)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < M.nIP)
    slot_inc[M.slot_pos[k]] = k;
}

// Weight of Gauss point g's value at local node n (ElementData
// integrationPointsToNode, ElHex8N3D.C:40-90, ElQua4NAx.C:37-58): the
// shape function of g's corner of the sub-element whose corners are the
// Gauss points (local coordinates +-1/sqrt3), evaluated at node n, i.e.
// prod_k (1 + sqrt3 s_k(n) s_k(g)) / 2 over the element's axes.  It depends
// only on the number m of axes on which n and g lie on the same side.
template <int NPE> __device__ __forceinline__ double extrapolation_weight(int n, int g)
{
  constexpr int DIM = NPE == 8 ? 3 : 2;
  const double r3 = 1.7320508075688772935; // sqrt(3)
  int m = 0;
#pragma unroll
  for (int k = 0; k < DIM; k++)
    m += node_sign(n, k) == node_sign(g, k);
  if constexpr (NPE == 8)
    return m == 3 ? (5.0 + 3.0 * r3) / 4 : m == 2 ? (-1.0 - r3) / 4 : m == 1 ? (-1.0 + r3) / 4 : (5.0 - 3.0 * r3) / 4;
  else
    return m == 2 ? 1.0 + r3 / 2 : m == 1 ? -0.5 : 1.0 - r3 / 2;
}

// Nodal values of point-state quantities as the reference extracts them for
// its node fields and result files (Node::fieldScalar / fieldSymTensor2,
// Node.C:244-365): at node i, the sum over its elements (in element order)
// and their Gauss points of extrapolation_weight * value, divided by the
// number of elements.  comps.c[j]: a point-state component DNL_IP_*, or
// DNL_NODE_AVG_VON_MISES (the von Mises stress of each point, dnlVonMises,
// Macros.h:71).  One thread per (component, node); dst [comps.n][nN].
struct AvgComps
{
  static constexpr int MAX = 32;
  int n;
  int c[MAX];
};
template <typename R, int NPE>
__global__ void k_node_average(DevModel M, const int *slot_inc, AvgComps comps, double *dst, const int *perm)
{
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)comps.n * M.nN)
    return;
  const int j = (int)(t / M.nN), i = (int)(t % M.nN); // i: the caller's node
  const int comp = comps.c[j];
  const int ni = perm ? perm[i] : i;
  const int kb = slot_begin(M, ni), ke = kb + M.csr_off[ni + 1] - M.csr_off[ni];
  double acc = 0.0;
  for (int k = kb; k < ke; k++)
  {
    const int inc = slot_inc[k];
    const int e = inc / NPE, loc = inc % NPE;
#pragma unroll
    for (int g = 0; g < NPE; g++)
    {
      const int q = e * NPE + g;
      double v;
      if (comp == DNL_NODE_AVG_VON_MISES)
      {
        const double s1 = ipv<R>(M, DNL_IP_STRESS + 0, q), s2 = ipv<R>(M, DNL_IP_STRESS + 3, q),
                     s3 = ipv<R>(M, DNL_IP_STRESS + 5, q), s4 = ipv<R>(M, DNL_IP_STRESS + 1, q),
                     s5 = ipv<R>(M, DNL_IP_STRESS + 2, q), s6 = ipv<R>(M, DNL_IP_STRESS + 4, q);
        v = sqrt(((s1 - s2) * (s1 - s2) + (s1 - s3) * (s1 - s3) + (s2 - s3) * (s2 - s3) +
                  6.0 * (s4 * s4 + s5 * s5 + s6 * s6)) / 2);
      }
      else
        v = (double)ipv<R>(M, comp, q);
      acc = __dadd_rn(acc, __dmul_rn(extrapolation_weight<NPE>(loc, g), v));
    }
  }
  dst[t] = acc / (double)(ke - kb);
}

// Components [c0, c0 + nc) of the point state, tile-major in R, to a
// component-major FP64 array (the layout of dnl_engine_get_ips).
template <typename R> __global__ void k_ips_out(DevModel M, int c0, int nc, double *dst)
{
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (long long)nc * M.nIP)
    return;
  const int c = c0 + (int)(k / M.nIP), q = (int)(k % M.nIP);
  dst[k] = (double)ipv<R>(M, c, q);
}

// The whole point state, tile-major in R, to a component-major array in R.
template <typename R> __global__ void k_ips_out_native(DevModel M, R *dst)
{
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (long long)DNL_IP_NCOMP * M.nIP)
    return;
  const int c = (int)(k / M.nIP), q = (int)(k % M.nIP);
  dst[k] = ipv<R>(M, c, q);
}

// --------------------------------------------------------- history items

// One thread per item (DNL_ITEM_*): the selected nodal vector, point state or
// kinetic energy copied to its place in `out` (offsets precomputed).
// kin holds the energies of every instance (3 per instance, kinetic first)
// on the field0 speeds, then on the field1 speeds.
template <typename R>
__global__ void k_gather_items(DevModel M, const int4 *items, const long long *off, int n, const double *kin,
                               double *out)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n)
    return;
  const int4 it = items[k];
  double *o = out + off[k];
  if (it.x == DNL_ITEM_POINT)
  {
    for (int c = 0; c < DNL_IP_NCOMP; c++)
      o[c] = (double)ipv<R>(M, c, it.z);
    return;
  }
  if (it.x == DNL_ITEM_KINETIC)
  {
    o[0] = kin[3 * ((it.y == DNL_NODE_SPEED_PREV ? M.nInst : 0) + it.z)];
    return;
  }
  const double4 v = node_vec(M, it.y, it.z);
  o[0] = v.x;
  o[1] = v.y;
  o[2] = v.z;
}

// ----------------------------------------------------- history records

// History records kept on the device while a single model runs: the save
// rule of HistoryFile::save (HistoryFile.C:292-317) per schedule j — a
// record is due when !(t > start_j && t < next_j), and next_j then moves on by
// save_j — evaluated at the end of every increment, after the time update, as
// Explicit::endStep calls Model::writeHistoryFiles (Explicit.C:539-552).
// A due increment appends one record of HIST_HEAD header words (time,
// increment, the increment's time step, the 64-bit mask of the due
// schedules as two 32-bit halves) and the values of the registered items.
constexpr int HIST_HEAD = DNL_HIST_HEAD;
struct HistRing
{
  int nSched, cap;
  double *start, *next, *save; // [nSched]
  int *count;                  // records since the last drain
  int *overflow;               // set when a record found the ring full
  long long *last;             // last increment checked
  double *rec;                 // [cap][HIST_HEAD + nValues]
};

// Kinetic energy of instance 0 on speed buffer fsel: the loop and tree of
// k_energies (same order, same bits).  Called by a whole block of 256.
__device__ __forceinline__ double block_kinetic(const DevModel &M, int fsel, double *sh)
{
  const Ctl &c = M.ctl[0];
  double ke = 0.0;
  for (int i = c.node_begin + threadIdx.x; i < c.node_end; i += blockDim.x)
  {
    const double4 v = M.v[fsel][i];
    ke += M.mass[i] * (v.x * v.x + v.y * v.y + v.z * v.z) / 2.0;
  }
  sh[threadIdx.x] = ke;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1)
  {
    if (threadIdx.x < s)
      sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

// One block of 256 after the end of the increment (single models).
template <typename R>
__global__ void __launch_bounds__(256) k_history_ring(DevModel M, HistRing H, const int4 *items,
                                                      const long long *off, int nItems, int nValues, int kin)
{
  pdl_wait();
  __shared__ double sh[256];
  __shared__ int slot;
  const Ctl &c = M.ctl[0];
  if (threadIdx.x == 0)
  {
    slot = -1;
    unsigned long long mask = 0ull;
    const long long committed = c.inc - ((c.prepared && c.active) ? 1 : 0);
    if (committed != *H.last)
    {
      *H.last = committed;
      const double t = c.t;
      for (int j = 0; j < H.nSched; j++)
        if (!(t > H.start[j] && t < H.next[j]))
        {
          H.next[j] += H.save[j];
          mask |= 1ull << j;
        }
      if (mask)
      {
        const int k = *H.count;
        if (k < H.cap)
        {
          slot = k;
          *H.count = k + 1;
          double *r = H.rec + (size_t)k * (HIST_HEAD + nValues);
          r[0] = t;
          r[1] = (double)committed;
          r[2] = c.dt_last;
          r[3] = (double)(unsigned)(mask & 0xffffffffull);
          r[4] = (double)(unsigned)(mask >> 32);
        }
        else
          *H.overflow = 1;
      }
    }
  }
  __syncthreads();
  if (slot < 0)
    return;
  double kinv[2] = {0.0, 0.0};
  if (kin)
  {
    kinv[0] = block_kinetic(M, c.f0, sh);
    kinv[1] = block_kinetic(M, 1 - c.f0, sh);
  }
  double *vals = H.rec + (size_t)slot * (HIST_HEAD + nValues) + HIST_HEAD;
  for (int k = threadIdx.x; k < nItems; k += blockDim.x)
  {
    const int4 it = items[k];
    double *o = vals + off[k];
    if (it.x == DNL_ITEM_POINT)
      for (int q = 0; q < DNL_IP_NCOMP; q++)
        o[q] = (double)ipv<R>(M, q, it.z);
    else if (it.x == DNL_ITEM_KINETIC)
      o[0] = kinv[it.y == DNL_NODE_SPEED_PREV ? 1 : 0];
    else
    {
      const double4 v = node_vec(M, it.y, it.z);
      o[0] = v.x;
      o[1] = v.y;
      o[2] = v.z;
    }
  }
}

// -------------------------------------------------------------- energies

// One block per instance, fixed-order tree sums (deterministic).
template <typename R, int NPE>
__global__ void k_energies(DevModel M, double *out /* [nInst*3] */, int speed_field)
{
  const int inst = blockIdx.x;
  const Ctl &c = M.ctl[inst];
  __shared__ double sh[3][256];
  double ke = 0.0, ei = 0.0, ep = 0.0;
  const int fsel = speed_field ? (1 - c.f0) : c.f0;
  for (int i = c.node_begin + threadIdx.x; i < c.node_end; i += blockDim.x)
  {
    const double4 v = M.v[fsel][i];
    ke += M.mass[i] * (v.x * v.x + v.y * v.y + v.z * v.z) / 2.0;
  }
  const double wfac = (NPE == 4 && !c.plane) ? 6.28318530717958647692 : 1.0;
  for (int q = c.elem_begin * NPE + threadIdx.x; q < c.elem_end * NPE; q += blockDim.x)
  {
    const MatDev &mp = M.mat[M.emat[q / NPE]];
    const double w = mp.rho0 * (double)ipv<R>(M, DNL_IP_DETJ0, q) * wfac;
    ei += w * (double)ipv<R>(M, DNL_IP_EINT, q);
    ep += w * (double)ipv<R>(M, DNL_IP_EINEL, q);
  }
  sh[0][threadIdx.x] = ke;
  sh[1][threadIdx.x] = ei;
  sh[2][threadIdx.x] = ep;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1)
  {
    if (threadIdx.x < s)
      for (int k = 0; k < 3; k++)
        sh[k][threadIdx.x] += sh[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; k++)
      out[3 * inst + k] = sh[k][0];
}

} // namespace
} // namespace dnl
