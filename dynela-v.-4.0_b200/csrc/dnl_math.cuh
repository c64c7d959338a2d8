// dnl_math.cuh - device tensor algebra, polar decomposition and the
// Johnson-Cook J2 radial return of the DynELA hot path, templated on the
// arithmetic type (double for the FP64 path, float for the mixed path).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "dnlgpu.h"

namespace dnl
{

template <typename R> struct Num;
template <> struct Num<double>
{
  static __device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
  static __device__ __forceinline__ double rsqrt_(double x) { return rsqrt(x); }
  static __device__ __forceinline__ double log_(double x) { return log(x); }
  static __device__ __forceinline__ double log1p_(double x) { return log1p(x); }
  static __device__ __forceinline__ double pow_(double x, double y) { return pow(x, y); }
  static __device__ __forceinline__ double abs_(double x) { return fabs(x); }
  static __device__ __forceinline__ double div_(double a, double b) { return a / b; }
  static constexpr double eps = 2.220446049250313e-16;
};
template <> struct Num<float>
{
  static __device__ __forceinline__ float sqrt_(float x) { return sqrtf(x); }
  static __device__ __forceinline__ float rsqrt_(float x) { return rsqrtf(x); }
  static __device__ __forceinline__ float log_(float x) { return __logf(x); }
  static __device__ __forceinline__ float log1p_(float x) { return log1pf(x); }
  // x^y for x > 0 through the fast base-2 exponential and logarithm
  static __device__ __forceinline__ float pow_(float x, float y) { return exp2f(y * __log2f(x)); }
  static __device__ __forceinline__ float abs_(float x) { return fabsf(x); }
  static __device__ __forceinline__ float div_(float a, float b) { return __fdividef(a, b); }
  static constexpr float eps = 1.1920929e-7f;
};

// symmetric storage xx, xy, xz, yy, yz, zz (SymTensor2 _data order)
__host__ __device__ constexpr int sym_index(int i, int j)
{
  return (i == j) ? (i == 0 ? 0 : (i == 1 ? 3 : 5)) : ((i + j) == 1 ? 1 : ((i + j) == 2 ? 2 : 4));
}

template <typename R> struct Sym
{
  R v[6];
};

template <typename R> __device__ __forceinline__ R sym_norm(const R s[6])
{
  return Num<R>::sqrt_(s[0] * s[0] + s[3] * s[3] + s[5] * s[5] + R(2) * (s[1] * s[1] + s[2] * s[2] + s[4] * s[4]));
}

template <typename R> __device__ __forceinline__ R sym_ddot(const R a[6], const R b[6])
{
  return a[0] * b[0] + a[3] * b[3] + a[5] * b[5] + R(2) * (a[1] * b[1] + a[2] * b[2] + a[4] * b[4]);
}

// S <- Q S Q^T for a full 3x3 Q (row-major) and symmetric S (SymTensor2::dotRxRT).
template <typename R> __device__ __forceinline__ void rotate_sym(const R Q[9], R S[6])
{
  R T[9]; // T = Q S
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
      T[3 * i + j] = Q[3 * i] * S[sym_index(0, j)] + Q[3 * i + 1] * S[sym_index(1, j)] + Q[3 * i + 2] * S[sym_index(2, j)];
  R out[6];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = i; j < 3; j++)
      out[sym_index(i, j)] = T[3 * i] * Q[3 * j] + T[3 * i + 1] * Q[3 * j + 1] + T[3 * i + 2] * Q[3 * j + 2];
#pragma unroll
  for (int k = 0; k < 6; k++)
    S[k] = out[k];
}

// Q S Q^T of two symmetric tensors at once; in FP32 as packed pairs
// (fma.rn.f32x2), the same arithmetic as rotate_sym on each.
template <typename R> __device__ __forceinline__ void rotate_sym2(const R Q[9], R S1[6], R S2[6])
{
  if constexpr (sizeof(R) == 4)
  {
    float2 S[6], QB[9];
#pragma unroll
    for (int k = 0; k < 6; k++)
      S[k] = make_float2(S1[k], S2[k]);
#pragma unroll
    for (int k = 0; k < 9; k++)
      QB[k] = make_float2(Q[k], Q[k]);
    float2 T[9];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++)
        T[3 * i + j] = __ffma2_rn(QB[3 * i + 2], S[sym_index(2, j)],
                                  __ffma2_rn(QB[3 * i + 1], S[sym_index(1, j)], __fmul2_rn(QB[3 * i], S[sym_index(0, j)])));
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = i; j < 3; j++)
      {
        const float2 o = __ffma2_rn(T[3 * i + 2], QB[3 * j + 2],
                                    __ffma2_rn(T[3 * i + 1], QB[3 * j + 1], __fmul2_rn(T[3 * i], QB[3 * j])));
        S1[sym_index(i, j)] = o.x;
        S2[sym_index(i, j)] = o.y;
      }
  }
  else
  {
    rotate_sym<R>(Q, S1);
    rotate_sym<R>(Q, S2);
  }
}

// One Jacobi rotation zeroing A(p, q) of the symmetric matrix held in A6,
// accumulated into the eigenvector matrix V (columns).
template <typename R, int P, int Q>
__device__ __forceinline__ void jacobi_rotate(R A[3][3], R V[3][3])
{
  R apq = A[P][Q];
  if (apq == R(0))
    return;
  R theta = (A[Q][Q] - A[P][P]) / (R(2) * apq);
  R at = Num<R>::abs_(theta);
  R t;
  if (at > R(1e18))
    t = R(0.5) / theta;
  else
    t = (theta >= R(0) ? R(1) : R(-1)) / (at + Num<R>::sqrt_(theta * theta + R(1)));
  R c = Num<R>::rsqrt_(t * t + R(1));
  R s = t * c;
#pragma unroll
  for (int r = 0; r < 3; r++)
  {
    R arp = A[r][P], arq = A[r][Q];
    A[r][P] = c * arp - s * arq;
    A[r][Q] = s * arp + c * arq;
  }
#pragma unroll
  for (int r = 0; r < 3; r++)
  {
    R apr = A[P][r], aqr = A[Q][r];
    A[P][r] = c * apr - s * aqr;
    A[Q][r] = s * apr + c * aqr;
  }
  A[P][Q] = A[Q][P] = R(0);
#pragma unroll
  for (int r = 0; r < 3; r++)
  {
    R vrp = V[r][P], vrq = V[r][Q];
    V[r][P] = c * vrp - s * vrq;
    V[r][Q] = s * vrp + c * vrq;
  }
}

// Cyclic Jacobi eigen-decomposition of a symmetric 3x3 matrix (Golub & Van
// Loan, Matrix Computations, sec. 8.5).  mu receives the eigenvalues, the
// columns of V the eigenvectors.
template <typename R> __device__ __forceinline__ void sym_eigen3(const R a6[6], R mu[3], R V[3][3])
{
  R A[3][3];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
    {
      A[i][j] = a6[sym_index(i, j)];
      V[i][j] = (i == j) ? R(1) : R(0);
    }
  // stop once the off-diagonal part is at the rounding level of the diagonal
  const R tol = Num<R>::eps;
  for (int sweep = 0; sweep < 12; sweep++)
  {
    R off = Num<R>::abs_(A[0][1]) + Num<R>::abs_(A[0][2]) + Num<R>::abs_(A[1][2]);
    R scale = Num<R>::abs_(A[0][0]) + Num<R>::abs_(A[1][1]) + Num<R>::abs_(A[2][2]) + off;
    if (off <= tol * scale)
      break;
    jacobi_rotate<R, 0, 1>(A, V);
    jacobi_rotate<R, 0, 2>(A, V);
    jacobi_rotate<R, 1, 2>(A, V);
  }
  mu[0] = A[0][0];
  mu[1] = A[1][1];
  mu[2] = A[2][2];
}

// Spectral functions of the small symmetric A = C - I (C = F^T F) by cyclic
// Jacobi: lnU = sum log1p(mu_k)/2 n_k n_k, Wm = U^-1 - I = sum ((1+mu_k)^-1/2 - 1) n_k n_k.
template <typename R> struct Spectral
{
  R lnU[6], Wm[6];
};
template <typename R>
__device__ __noinline__ Spectral<R> spectral_jacobi(R a0, R a1, R a2, R a3, R a4, R a5)
{
  const R A[6] = {a0, a1, a2, a3, a4, a5};
  Spectral<R> out;
  R *lnU = out.lnU, *Wm = out.Wm;
  R mu[3], V[3][3];
  sym_eigen3<R>(A, mu, V);
  R hl[3], g[3];
#pragma unroll
  for (int k = 0; k < 3; k++)
  {
    hl[k] = R(0.5) * Num<R>::log1p_(mu[k]);
    g[k] = Num<R>::rsqrt_(R(1) + mu[k]) - R(1);
  }
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = i; j < 3; j++)
    {
      R a = R(0), b = R(0);
#pragma unroll
      for (int k = 0; k < 3; k++)
      {
        R p = V[i][k] * V[j][k];
        a += hl[k] * p;
        b += g[k] * p;
      }
      lnU[sym_index(i, j)] = a;
      Wm[sym_index(i, j)] = b;
    }
  return out;
}

// The same two functions as power series, without eigenvectors.  By
// Cayley-Hamilton every power is A^k = al I + be A + ga A^2 with the scalar
// recurrence A^(k+1) = (ga I3) I + (al - ga I2) A + (be + ga I1) A^2 (I1, I2,
// I3 the invariants of A), so both series cost a few scalar operations per
// term:  log(1+x) = sum (-1)^(k+1) x^k / k,  (1+x)^-1/2 - 1 = sum binom(-1/2, k) x^k.
// The series stop when |A|_F^k falls below the rounding level; returns false
// when |A|_F is too large for a short series (the caller then uses Jacobi).
template <typename R> struct SeriesCoef
{
  R log1p[64];   // term k: (-1)^(k+1) / k              (index k, entry 0 unused)
  R invsqrt[64]; // term k: binom(-1/2, k) = (-1)^k (2k-1)!! / (2k)!!
};
template <typename R> __host__ __device__ constexpr SeriesCoef<R> series_coef()
{
  SeriesCoef<R> c{};
  double w = 1.0;
  for (int k = 1; k < 64; k++)
  {
    c.log1p[k] = R(((k & 1) ? 1.0 : -1.0) / k);
    w *= -(2.0 * k - 1.0) / (2.0 * k);
    c.invsqrt[k] = R(w);
  }
  return c;
}
// indexed by the unrolled loop counter: compile-time offsets into the constant bank
static __constant__ SeriesCoef<float> c_series_f = series_coef<float>();
static __constant__ SeriesCoef<double> c_series_d = series_coef<double>();

template <typename R> __device__ __forceinline__ bool spectral_series(const R A[6], R lnU[6], R Wm[6])
{
  const SeriesCoef<R> &co = [] () -> const SeriesCoef<R> & {
    if constexpr (sizeof(R) == 4)
      return c_series_f;
    else
      return c_series_d;
  }();
  const bool fp64 = sizeof(R) == 8;
  const R r = Num<R>::sqrt_(A[0] * A[0] + A[3] * A[3] + A[5] * A[5] + R(2) * (A[1] * A[1] + A[2] * A[2] + A[4] * A[4]));
  const R rmax = fp64 ? R(0.25) : R(0.35);
  if (!(r < rmax))
    return false;
  const R tol = fp64 ? R(2e-17) : R(3e-8);
  const R I1 = A[0] + A[3] + A[5];
  const R I2 = A[0] * A[3] + A[3] * A[5] + A[5] * A[0] - A[1] * A[1] - A[2] * A[2] - A[4] * A[4];
  const R I3 = A[0] * (A[3] * A[5] - A[4] * A[4]) - A[1] * (A[1] * A[5] - A[4] * A[2]) + A[2] * (A[1] * A[4] - A[3] * A[2]);
  R al = R(0), be = R(1), ga = R(0);      // A^1
  R l0 = R(0), l1 = R(0), l2 = R(0);      // log(I + A)
  R w0 = R(0), w1 = R(0), w2 = R(0);      // (I + A)^-1/2 - I
  R rk = r;
  // r < rmax bounds the terms the series needs (r^k < tol by k = 17 in FP32,
  // 28 in FP64): unrolled, the coefficients are constant-bank operands
  constexpr int KMAX = sizeof(R) == 4 ? 20 : 32;
#pragma unroll
  for (int k = 1; k < KMAX; k++)
  {
    const R cl = co.log1p[k], cw = co.invsqrt[k];
    l0 += cl * al;
    l1 += cl * be;
    l2 += cl * ga;
    w0 += cw * al;
    w1 += cw * be;
    w2 += cw * ga;
    if (rk < tol)
      break;
    const R nal = ga * I3, nbe = al - ga * I2, nga = be + ga * I1;
    al = nal;
    be = nbe;
    ga = nga;
    rk *= r;
  }
  // A^2
  R A2[6];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = i; j < 3; j++)
      A2[sym_index(i, j)] = A[sym_index(i, 0)] * A[sym_index(0, j)] + A[sym_index(i, 1)] * A[sym_index(1, j)] +
                            A[sym_index(i, 2)] * A[sym_index(2, j)];
#pragma unroll
  for (int c = 0; c < 6; c++)
  {
    const R d = (c == 0 || c == 3 || c == 5) ? R(1) : R(0);
    lnU[c] = R(0.5) * (l0 * d + l1 * A[c] + l2 * A2[c]);
    Wm[c] = w0 * d + w1 * A[c] + w2 * A2[c];
  }
  return true;
}

// Polar decomposition F = R U of F = I + H and the logarithmic strain
// increment ln U (Tensor2::polarCuppenLnU, Tensor2.C:1237-1457, restated):
// with A = F^T F - I = H + H^T + H^T H, ln U = log(I + A)/2 and
// R = F U^-1, U^-1 = (I + A)^-1/2.  Working on A keeps the relative precision
// of the small increments; the series above is used when |A| is small, the
// Jacobi eigen-decomposition otherwise.
template <typename R> __device__ __forceinline__ void polar_lnU(const R H[9], R lnU[6], R Rot[9])
{
  R A[6];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = i; j < 3; j++)
      A[sym_index(i, j)] = H[3 * i + j] + H[3 * j + i] + H[i] * H[j] + H[3 + i] * H[3 + j] + H[6 + i] * H[6 + j];
  R Wm[6]; // U^-1 - I
  if (!spectral_series<R>(A, lnU, Wm))
  {
    // arguments and result by value: no array of this function's has its
    // address taken, so A, lnU and Wm stay in registers on the series path
    const Spectral<R> sp = spectral_jacobi<R>(A[0], A[1], A[2], A[3], A[4], A[5]);
#pragma unroll
    for (int c = 0; c < 6; c++)
    {
      lnU[c] = sp.lnU[c];
      Wm[c] = sp.Wm[c];
    }
  }
  // R = (I + H)(I + Wm) = I + H + Wm + H Wm
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
    {
      R s = H[3 * i + j] + Wm[sym_index(i, j)];
#pragma unroll
      for (int k = 0; k < 3; k++)
        s += H[3 * i + k] * Wm[sym_index(k, j)];
      Rot[3 * i + j] = s + ((i == j) ? R(1) : R(0));
    }
}

// Johnson-Cook parameters of one material in the precision a return runs in.
template <typename R> struct JCParams
{
  R A, B, C, n, m, depsp0, Tm, Tref, invTmT, thermal; // invTmT = 1/(Tm-Tref), thermal = tq/(rho0 Cp)
  R twoG, invRho0, K;                                 // 2G, 1/rho0 and the bulk modulus of the return
};

// Material constants (Material.h, JohnsonCookLaw.C:132-143) with the derived
// ones the return uses, and the Johnson-Cook block in FP64 and in FP32.
struct MatDev
{
  double young, poisson, rho0, cp, tq, T0;
  double A, B, C, n, m, depsp0, Tm, Tref;
  double twoG, K, heatFrac, wave2; // E/(1+nu), E/(3(1-2nu)), tq/(rho0 Cp), E(1-nu)/((1+nu)(1-2nu))
  JCParams<double> jc64;
  JCParams<float> jc32;
};

// Host: the device copy of a material description.
inline MatDev make_mat(const dnl_material &m)
{
  MatDev d;
  d.young = m.young;
  d.poisson = m.poisson;
  d.rho0 = m.density;
  d.cp = m.heat_capacity;
  d.tq = m.taylor_quinney;
  d.T0 = m.T0;
  d.A = m.A;
  d.B = m.B;
  d.C = m.C;
  d.n = m.n;
  d.m = m.m;
  d.depsp0 = m.depsp0;
  d.Tm = m.Tm;
  d.Tref = m.Tref;
  d.twoG = m.young / (1.0 + m.poisson);                          // Material.h:110-114
  d.K = m.young / (3.0 * (1.0 - 2.0 * m.poisson));               // Material.h:152-156
  d.heatFrac = m.taylor_quinney / (m.density * m.heat_capacity); // Material.h:165-169
  d.wave2 = m.young * (1.0 - m.poisson) / ((1.0 + m.poisson) * (1.0 - 2.0 * m.poisson)); // Element.C:358
  d.jc64 = {d.A, d.B, d.C, d.n, d.m, d.depsp0, d.Tm, d.Tref, 1.0 / (d.Tm - d.Tref), d.heatFrac, d.twoG,
            1.0 / d.rho0, d.K};
  d.jc32 = {(float)d.A,    (float)d.B,      (float)d.C,    (float)d.n,           (float)d.m,
            (float)d.depsp0, (float)d.Tm,   (float)d.Tref, (float)d.jc64.invTmT, (float)d.heatFrac,
            (float)d.twoG, (float)(1.0 / d.rho0), (float)d.K};
  return d;
}

// The Johnson-Cook law as the return calls it.  The parameters are read from
// the material at each use instead of being held in registers through the
// return (the element pass is limited by registers).  PARAM false: q points to
// the material in global memory (read-only loads of one cached line that every
// thread shares); PARAM true: q points into the kernel's parameter block (a
// model with one material: DevModel::one32 / one64), whose values the
// arithmetic takes as constant-bank operands, without a load.
template <typename R, bool PARAM = false> struct JC
{
  const JCParams<R> *q;
  __device__ __forceinline__ R ld(const R &v) const
  {
    if constexpr (PARAM)
      return v;
    else
      return __ldg(&v);
  }
  __device__ __forceinline__ void load(const MatDev &p)
  {
    if constexpr (sizeof(R) == 4)
      q = &p.jc32;
    else
      q = &p.jc64;
  }
  __device__ __forceinline__ R twoG() const { return ld(q->twoG); }
  __device__ __forceinline__ R heatFrac() const { return ld(q->thermal); }
  __device__ __forceinline__ R invRho0() const { return ld(q->invRho0); }
  __device__ __forceinline__ R K() const { return ld(q->K); }
  // JohnsonCookLaw::getYieldStress (JohnsonCookLaw.C:146-170) and the analytic
  // total derivative getDerivateYieldStress (JohnsonCookLaw.C:298-339), in one pass.
  __device__ __forceinline__ void eval(R epsp, R depsp, R T, R dt, R &yield, R &hard, bool wantHard) const
  {
    R pn = Num<R>::pow_(epsp, ld(q->n)); // epsp^n
    R hard0 = ld(q->A) + ld(q->B) * pn;
    bool rate = depsp > ld(q->depsp0);
    R visc0 = rate ? R(1) + ld(q->C) * Num<R>::log_(depsp / ld(q->depsp0)) : R(1);
    R temp0 = R(1), temp1 = R(0);
    bool hot = T > ld(q->Tref), melt = !(T < ld(q->Tm));
    if (hot)
    {
      if (!melt)
      {
        temp1 = Num<R>::pow_((T - ld(q->Tref)) * ld(q->invTmT), ld(q->m));
        temp0 = R(1) - temp1;
      }
      else
        temp0 = R(0);
    }
    yield = hard0 * visc0 * temp0;
    if (wantHard)
    {
      R h = ld(q->n) * ld(q->B) * (epsp > R(0) ? pn / epsp : R(0)) * visc0 * temp0; // n B epsp^(n-1) ...
      if (rate)
        h += hard0 * ld(q->C) * temp0 / (depsp * dt);
      if (hot && !melt)
        h -= ld(q->m) * ld(q->thermal) * hard0 * hard0 * visc0 * visc0 * temp0 * temp1 / (T - ld(q->Tref));
      hard = h;
    }
  }
};

// Per-point state handled by the radial return.  The plastic strain tensor is
// not carried: its increment is kplast times the deviator of the returned
// stress (gamma s*/|s*| = gamma/(|s*| - 2G gamma) s_new, Element.C:587-590).
template <typename R> struct ReturnState
{
  R s[6]; // stress (in: old, out: new, before the final rotation)
  R epsp, depsp, gamma, gcum, yield, T, pressure, eint, einel;
  R kplast; // out: plastic strain increment / deviator of the new stress (0 if elastic)
};

// Trial equivalent stress sqrt(3/2)|dev(sigma_old) + 2G dev(dE)| and the yield
// stress the return starts from (with the reference's lazy first evaluation at
// gamma = 1e-8, Element.C:458-463): the inputs of the learned initial guess.
template <typename R, class Law>
__device__ __forceinline__ void trial_state(const Law &jc, R twoG, const R dE[6], const ReturnState<R> &st, R dt,
                                            R &Strial, R &yield0)
{
  R p0 = (st.s[0] + st.s[3] + st.s[5]) / R(3), pe = (dE[0] + dE[3] + dE[5]) / R(3);
  R d[6];
#pragma unroll
  for (int c = 0; c < 6; c++)
    d[c] = st.s[c] + twoG * dE[c];
  d[0] -= p0 + twoG * pe;
  d[3] -= p0 + twoG * pe;
  d[5] -= p0 + twoG * pe;
  Strial = R(1.2247448713915890491) * sym_norm(d);
  yield0 = st.yield;
  if (yield0 == R(0))
  {
    R dummy;
    jc.eval(R(1e-8), R(1e-8) / dt, st.T, dt, yield0, dummy, false);
  }
}

// Element::computeStress (Element.C:407-622) for one integration point.  The
// Newton-bisection iteration on gamma is the reference's; tolNR = 1e-8 and
// itMax = 250 for FP64.  For FP32 the step tolerance is widened to a few ulp
// of gamma and `ok` is cleared when the iteration fails to converge in 60
// steps or the final residual test |f| <= 1e-5 Strial + 2 f' tol fails; the
// caller then re-solves the point in FP64.
// A non-negative gamma0 replaces the warm start (the previous increment's gamma)
// as the first iterate; the bracket and the stopping tests are unchanged.
// Returns the number of yield-function evaluations of the iteration (0 for an
// elastic point).
// direct: Element::computeStressDirect (Element.C:625-850) instead, one step
// gamma = (|s*| - sqrt(2/3) sigma_y) / (2G (1 + h / (3G))) with the slope h at
// the previous plastic strain (or 1e-8) and rate and the initial temperature,
// then the yield stress at the new state (1 evaluation).
template <typename R, class Law>
__device__ __forceinline__ int radial_return(const Law &jc, R twoG, R heatFrac, R inv_rho0, const R dE[6], R dt,
                                             ReturnState<R> &st, bool &ok, R gamma0 = R(-1), bool direct = false)
{
  const R SQ32 = R(1.2247448713915890491), SQ23 = R(0.81649658092772603273);
  const R gammaInitial = R(1e-8);
  const bool fp64 = sizeof(R) == 8;
  const int itMax = fp64 ? 250 : 60;
  R twoG32 = SQ32 * twoG;
  R dev[6];
  // dE : sigma_old, the first half of the stress power (Element.C:608)
  const R dEsOld = sym_ddot(dE, st.s);
  R p0 = (st.s[0] + st.s[3] + st.s[5]) / R(3);
#pragma unroll
  for (int c = 0; c < 6; c++)
    dev[c] = st.s[c];
  dev[0] -= p0;
  dev[3] -= p0;
  dev[5] -= p0;
  R Snorm0 = sym_norm(dev);
  R pe = (dE[0] + dE[3] + dE[5]) / R(3);
  dev[0] += twoG * (dE[0] - pe);
  dev[1] += twoG * dE[1];
  dev[2] += twoG * dE[2];
  dev[3] += twoG * (dE[3] - pe);
  dev[4] += twoG * dE[4];
  dev[5] += twoG * (dE[5] - pe);
  R Snorm = sym_norm(dev);
  R Strial = SQ32 * Snorm;
  R T0 = st.T, T = T0;
  R epsp0 = st.epsp;
  R gamma = R(0);
  R yield = st.yield;
  R dummy;
  int iterate = 0;
  ok = true;
  st.kplast = R(0);
  if (yield == R(0))
  {
    jc.eval(gammaInitial, gammaInitial / dt, T, dt, yield, dummy, false);
    st.yield = yield;
  }
  if (Strial > yield && direct)
  {
    R dummy, hard;
    jc.eval(epsp0 > R(0) ? epsp0 : gammaInitial, st.depsp, T0, dt, dummy, hard, true);
    gamma = (Snorm - SQ23 * yield) / (twoG * (R(1) + hard / (R(1.5) * twoG)));
    const R depsp = SQ23 * gamma / dt, epsp = epsp0 + SQ23 * gamma;
    T = T0 + R(0.5) * gamma * heatFrac * (SQ23 * yield + Snorm0);
    jc.eval(epsp, depsp, T, dt, yield, dummy, false);
    const R invS = R(1) / Snorm;
    const R scale = R(1) - twoG * gamma * invS;
    st.kplast = gamma * invS / scale;
#pragma unroll
    for (int c = 0; c < 6; c++)
      dev[c] *= scale;
    st.epsp = epsp;
    st.depsp = depsp;
    st.gamma = gamma;
    st.gcum += gamma;
    st.yield = yield;
    iterate = 1;
  }
  else if (Strial > yield)
  {
    R gammaMin = R(0);
    R gammaMax = (Strial - yield) / twoG32;
    gamma = st.gamma;
    if (epsp0 == R(0))
      gamma = SQ32 * gammaInitial;
    if (gamma0 >= R(0))
      gamma = gamma0;
    R depsp = SQ23 * gamma / dt;
    R epsp = epsp0 + SQ23 * gamma;
    T = T0 + R(0.5) * gamma * heatFrac * (SQ23 * yield + Snorm0);
    R fun = R(0), dfun = twoG32, tol = R(1e-8);
    bool bisected = false; // the last step halved the bracket instead of a Newton step
    for (;;)
    {
      R hard;
      jc.eval(epsp, depsp, T, dt, yield, hard, true);
      fun = Strial - gamma * twoG32 - yield;
      if (fun < R(0))
        gammaMax = gamma;
      else
        gammaMin = gamma;
      dfun = twoG32 + SQ23 * hard;
      R dgamma = fun / dfun;
      gamma += dgamma;
      bisected = (gammaMax - gamma) * (gamma - gammaMin) < R(0);
      if (bisected)
      {
        dgamma = R(0.5) * (gammaMax - gammaMin);
        gamma = gammaMin + dgamma;
      }
      R tolRel = R(4) * Num<R>::eps * Num<R>::abs_(gamma);
      tol = (fp64 || tolRel < R(1e-8)) ? R(1e-8) : tolRel;
      if (Num<R>::abs_(dgamma) < tol)
        break;
      depsp = SQ23 * gamma / dt;
      epsp = epsp0 + SQ23 * gamma;
      T = T0 + R(0.5) * gamma * heatFrac * (SQ23 * yield + Snorm0);
      iterate += 1;
      if (iterate > itMax || !(gamma == gamma))
      {
        ok = false;
        return iterate + 1;
      }
    }
    // FP32 acceptance: after a Newton step the last residual is the one before
    // that step, so it is bounded by dfun times the step tolerance; a rounding
    // failure shows there.  An exit by halving the bracket (Element.C:539-547:
    // the bracket closed to the step tolerance, with a residual that can reach
    // a few MPa) is the algorithm's own exit: from the reference's start the
    // FP64 iteration ends those points in the same bracket, after as many
    // steps, with the same residual, so re-solving them in FP64 changes
    // nothing but costs time.  Where the bracket closes depends on the start,
    // so a point started from a guess (gamma0) that ends that way is still
    // re-solved, from the reference's start.
    if (!fp64 && !(bisected && gamma0 < R(0)) && !(Num<R>::abs_(fun) <= R(1e-5) * Strial + R(2) * dfun * tol))
    {
      ok = false;
      return iterate + 1;
    }
    iterate += 1;
    const R invS = R(1) / Snorm;
    const R scale = R(1) - twoG * gamma * invS;
    // plastic strain increment gamma dev*/Snorm = kplast * (scale dev*)
    st.kplast = gamma * invS / scale;
#pragma unroll
    for (int c = 0; c < 6; c++)
      dev[c] *= scale;
    st.epsp = epsp0 + SQ23 * gamma;
    st.depsp = SQ23 * gamma / dt;
    st.gamma = gamma;
    st.gcum += gamma;
    st.yield = yield;
  }
  R p = st.pressure;
  st.s[0] = dev[0] + p;
  st.s[1] = dev[1];
  st.s[2] = dev[2];
  st.s[3] = dev[3] + p;
  st.s[4] = dev[4];
  st.s[5] = dev[5] + p;
  st.eint += R(0.5) * (dEsOld + sym_ddot(dE, st.s)) * inv_rho0;
  if (gamma != R(0))
  {
    R plWorkInc = R(0.5) * gamma * (sym_norm(dev) + Snorm0);
    st.einel += plWorkInc * inv_rho0;
    st.T += heatFrac * plWorkInc;
  }
  return iterate;
}

} // namespace dnl
