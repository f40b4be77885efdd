// D3Q19 lattice, storage forms and the per-cell BGK collision shared by every
// kernel of the library.
//
// Velocity set and pull offsets: SRC/alloca.F90:57-175, SRC/col_MC.F90:113-131
// (population q of the reference is index q-1 here). Collision arithmetic:
// SRC/col_MC.F90:133-219,333-351 in the deviation form (cte1 = 1, cte0 = 0).
#pragma once
#include <cuda_fp16.h>
#include <cstdint>

namespace bgk {

constexpr int Q = 19;

// c_q of the reference velocity set, q = 1..19 -> index 0..18.
__host__ __device__ constexpr int cxq(int q) {
  return q < 5 ? 1 : (q < 9 ? 0 : (q < 14 ? -1 : 0));
}
__host__ __device__ constexpr int cyq(int q) {
  // -1 0 1 0 0 0 1 1 1 -1 0 1 0 0 0 -1 -1 -1 0
  return (q == 0 || q == 9 || q == 15 || q == 16 || q == 17) ? -1
         : (q == 2 || q == 6 || q == 7 || q == 8 || q == 11) ? 1 : 0;
}
__host__ __device__ constexpr int czq(int q) {
  // 0 -1 0 1 0 1 1 0 -1 0 -1 0 1 0 -1 -1 0 1 0
  return (q == 1 || q == 8 || q == 10 || q == 14 || q == 15) ? -1
         : (q == 3 || q == 5 || q == 6 || q == 12 || q == 17) ? 1 : 0;
}
// Populations that cross a z face: cz = +1 (q = 3, 5, 6, 12, 17; reference
// 4, 6, 7, 13, 18) and cz = -1 (q = 1, 8, 10, 14, 15; reference 2, 9, 11, 15,
// 16), the five per face that SRC/bcond.comm.step3.F90:77-297 exchanges.
// zslot(q) is the position of q in its list.
constexpr int NZF = 5;
__host__ __device__ constexpr int zslot(int q) {
  return (q == 3 || q == 1) ? 0 : (q == 5 || q == 8) ? 1 : (q == 6 || q == 10) ? 2 : (q == 12 || q == 14) ? 3 : 4;
}
// Opposite direction, c(opp q) = -c(q). Pairs in the reference's 1-based
// numbering: 1<->12, 2<->13, 3<->10, 4<->11, 5<->14, 6<->15, 7<->16, 8<->17,
// 9<->18, 19 fixed.
__host__ __device__ constexpr int oppq(int q) {
  return q == 18 ? 18 : (q < 9 ? (q == 0 ? 11 : q == 1 ? 12 : q == 2 ? 9 : q == 3 ? 10 : q == 4 ? 13 : q + 9)
                                  : (q == 9 ? 2 : q == 10 ? 3 : q == 11 ? 0 : q == 12 ? 1 : q == 13 ? 4 : q - 9));
}

// ---------------------------------------------------------------- arithmetic
// Ex<T> rounds every operation separately (no FMA contraction), so device
// results equal a host build that evaluates the same expressions in order.
template <class T> struct Ex { T v; };
__device__ __forceinline__ Ex<double> operator+(Ex<double> a, Ex<double> b) { return {__dadd_rn(a.v, b.v)}; }
__device__ __forceinline__ Ex<double> operator-(Ex<double> a, Ex<double> b) { return {__dsub_rn(a.v, b.v)}; }
__device__ __forceinline__ Ex<double> operator*(Ex<double> a, Ex<double> b) { return {__dmul_rn(a.v, b.v)}; }
__device__ __forceinline__ Ex<double> operator/(Ex<double> a, Ex<double> b) { return {__ddiv_rn(a.v, b.v)}; }
__device__ __forceinline__ Ex<float> operator+(Ex<float> a, Ex<float> b) { return {__fadd_rn(a.v, b.v)}; }
__device__ __forceinline__ Ex<float> operator-(Ex<float> a, Ex<float> b) { return {__fsub_rn(a.v, b.v)}; }
__device__ __forceinline__ Ex<float> operator*(Ex<float> a, Ex<float> b) { return {__fmul_rn(a.v, b.v)}; }
__device__ __forceinline__ Ex<float> operator/(Ex<float> a, Ex<float> b) { return {__fdiv_rn(a.v, b.v)}; }
template <class T> __device__ __forceinline__ Ex<T> operator-(Ex<T> a) { return {-a.v}; }
__device__ __forceinline__ Ex<double> esqrt(Ex<double> a) { return {__dsqrt_rn(a.v)}; }
__device__ __forceinline__ Ex<float> esqrt(Ex<float> a) { return {__fsqrt_rn(a.v)}; }

template <class V> struct Num;  // constants and conversions for V
template <> struct Num<double> {
  using R = double;
  __device__ static __forceinline__ double c(double x) { return x; }
  __device__ static __forceinline__ double raw(double x) { return x; }
  __device__ static __forceinline__ double wrap(double x) { return x; }
};
template <> struct Num<float> {
  using R = float;
  __device__ static __forceinline__ float c(double x) { return (float)x; }
  __device__ static __forceinline__ float raw(float x) { return x; }
  __device__ static __forceinline__ float wrap(float x) { return x; }
};
template <class T> struct Num<Ex<T>> {
  using R = T;
  __device__ static __forceinline__ Ex<T> c(double x) { return {(T)x}; }
  __device__ static __forceinline__ T raw(Ex<T> x) { return x.v; }
  __device__ static __forceinline__ Ex<T> wrap(T x) { return {x}; }
};

// ------------------------------------------------------------ storage forms
// Per-launch constants of the collision, for every form.
struct StepK {
  double omega;   // F64
  float omega_f;  // F32
  float inv;      // F16: 1/scale
  float om1;      // F16: 1 - omega
  float kw[3];    // F16: omega*scale*w for w = 1/3, 1/18, 1/36
  // Smagorinsky closure (SRC/col_MC.F90:221-309): les != 0 enables it;
  // cs18 = 18*cteS^2, tauh = 1/(2*omega), tau2 = (1/omega)^2, in double (F64)
  // and float (F32, F16) arithmetic
  int les;
  double cs18, tauh, tau2;
  float cs18_f, tauh_f, tau2_f;
  float scale;    // F16: scale
};

// Weight class of population q: 0 -> 1/3 (rest), 1 -> 1/18, 2 -> 1/36.
__host__ __device__ constexpr int wclass(int q) {
  return q == 18 ? 0 : ((q == 4 || q == 5 || q == 7 || q == 13 || q == 14 || q == 16) ? 1 : 2);
}

template <class V>
__device__ __forceinline__ void collide(V (&x)[Q], V omega);
template <class V>
__device__ __forceinline__ void collide_les(V (&x)[Q], V cs18, V tauh, V tau2);

// F64: double storage / double arithmetic (reference DOUBLE_P build).
// F32: float storage of f - w / float arithmetic (reference default build).
// Both use the reference's evaluation order with every operation rounded.
struct F64 {
  using S = double; using R = double; using V = Ex<double>;
  static constexpr int id = 0;
  __device__ static __forceinline__ R dec(S s, R) { return s; }
  __device__ static __forceinline__ S enc(R r, R) { return r; }
  template <bool LES = false>
  __device__ static __forceinline__ void cell(S (&s)[Q], const StepK& k) {
    V x[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) x[q] = V{s[q]};
    if constexpr (LES) collide_les<V>(x, V{k.cs18}, V{k.tauh}, V{k.tau2});
    else collide<V>(x, V{k.omega});
#pragma unroll
    for (int q = 0; q < Q; ++q) s[q] = x[q].v;
  }
};
struct F32 {
  using S = float; using R = float; using V = Ex<float>;
  static constexpr int id = 1;
  __device__ static __forceinline__ R dec(S s, R) { return s; }
  __device__ static __forceinline__ S enc(R r, R) { return r; }
  template <bool LES = false>
  __device__ static __forceinline__ void cell(S (&s)[Q], const StepK& k) {
    V x[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) x[q] = V{s[q]};
    if constexpr (LES) collide_les<V>(x, V{k.cs18_f}, V{k.tauh_f}, V{k.tau2_f});
    else collide<V>(x, V{k.omega_f});
#pragma unroll
    for (int q = 0; q < Q; ++q) s[q] = x[q].v;
  }
};

// F16: binary16 storage of y = scale*(f - w), float arithmetic. The FP16 form
// has no reference counterpart (SRC/precision.F90:40-43 stops on HALF_P), so
// its collision is written for this storage: it works on the scaled values y
// directly, keeps the density deviation dr = sum(f - w) apart from 1, treats
// each pair of opposite directions together and uses fused multiply-adds:
//   dr = sum(y)/scale, u = j(y)/(scale*(1 + dr)), a = -1.5|u|^2,
//   P(+-) = +-3 cu + 4.5 cu^2 + a for the pair (q, opp q), cu = c_q.u
//   (f_eq/w - 1 = dr + (1+dr) P), and
//   y' = (1 - omega) y + K dr + K (1 + dr) P, K = omega*scale*w,
// regrouped per weight class with kr = K + K dr:
//   t = (4.5 kr cu) cu + (kr a + K dr),  y'(+-) = (1 - omega) y + t +- 3 kr cu
// (six fused operations per pair). Sums and roundings are fixed (moments16,
// pair16) and restated by the oracle.
struct Mom16 { float dr, ux, uy, uz, a, kr3[3], kr45[3], kra[3]; };

__device__ __forceinline__ Mom16 moments16(const float (&y)[Q], const StepK& k) {
  const float sp = __fadd_rn(__fadd_rn(__fadd_rn(y[0], y[1]), __fadd_rn(y[2], y[3])), y[4]);
  const float sm = __fadd_rn(__fadd_rn(__fadd_rn(y[9], y[10]), __fadd_rn(y[11], y[12])), y[13]);
  const float s0 = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(y[5], y[6]), __fadd_rn(y[7], y[8])),
                                       __fadd_rn(__fadd_rn(y[14], y[15]), __fadd_rn(y[16], y[17]))),
                             y[18]);
  const float sum = __fadd_rn(__fadd_rn(sp, sm), s0);
  const float jx = __fsub_rn(sp, sm);
  const float jyp = __fadd_rn(__fadd_rn(__fadd_rn(y[2], y[6]), __fadd_rn(y[7], y[8])), y[11]);
  const float jym = __fadd_rn(__fadd_rn(__fadd_rn(y[0], y[9]), __fadd_rn(y[15], y[16])), y[17]);
  const float jzp = __fadd_rn(__fadd_rn(__fadd_rn(y[3], y[5]), __fadd_rn(y[6], y[12])), y[17]);
  const float jzm = __fadd_rn(__fadd_rn(__fadd_rn(y[1], y[8]), __fadd_rn(y[10], y[14])), y[15]);
  Mom16 m;
  const float dr = __fmul_rn(sum, k.inv);
  m.dr = dr;
  // inv/(1 + dr) as inv * rcp(1 + dr): inv is a power of two, so scaling the
  // correctly rounded reciprocal is exact and the result equals the division
  const float r = __fmul_rn(k.inv, __frcp_rn(__fadd_rn(1.0f, dr)));
  m.ux = __fmul_rn(jx, r);
  m.uy = __fmul_rn(__fsub_rn(jyp, jym), r);
  m.uz = __fmul_rn(__fsub_rn(jzp, jzm), r);
  const float usq = __fmaf_rn(m.uz, m.uz, __fmaf_rn(m.uy, m.uy, __fmul_rn(m.ux, m.ux)));
  m.a = __fmul_rn(-1.5f, usq);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float kd = __fmul_rn(k.kw[c], dr);
    const float kr = __fadd_rn(k.kw[c], kd);
    m.kr3[c] = __fmul_rn(3.0f, kr);
    m.kr45[c] = __fmul_rn(4.5f, kr);
    m.kra[c] = __fmaf_rn(kr, m.a, kd);
  }
  return m;
}

// c_q.u: the first non-zero component, plus the second one if any.
__device__ __forceinline__ float cdotu(int q, const Mom16& m) {
  const int cx = cxq(q), cy = cyq(q), cz = czq(q);
  float cu = 0.0f;
  bool first = true;
  if (cx != 0) { cu = cx > 0 ? m.ux : -m.ux; first = false; }
  if (cy != 0) { const float t = cy > 0 ? m.uy : -m.uy; cu = first ? t : __fadd_rn(cu, t); first = false; }
  if (cz != 0) { const float t = cz > 0 ? m.uz : -m.uz; cu = first ? t : __fadd_rn(cu, t); }
  return cu;
}

// Post-collision scaled values of the pair (q, opp q), q in 0..8.
__device__ __forceinline__ void pair16(int q, float yq, float yo, const Mom16& m, float om1, float& oq, float& oo) {
  const int c = wclass(q);
  const float cu = cdotu(q, m);
  const float t = __fmaf_rn(__fmul_rn(m.kr45[c], cu), cu, m.kra[c]);
  oq = __fmaf_rn(m.kr3[c], cu, __fmaf_rn(om1, yq, t));
  oo = __fmaf_rn(-m.kr3[c], cu, __fmaf_rn(om1, yo, t));
}

// Rest population (cu = 0, P = a).
__device__ __forceinline__ float rest16(float y, const Mom16& m, float om1) {
  return __fmaf_rn(om1, y, m.kra[0]);
}

// FP16 form with the Smagorinsky closure: the sums, dr, u and a of
// moments16; Pi_neq from the second moments of the stored values minus the
// equilibrium's closed form (D3Q19: sum_q c_a c_b (f_eq - w)_q =
// dr delta_ab / 3 + rho u_a u_b, rho = 1 + dr), Ptotal = sqrt(Pi:Pi),
// tau = tauh + sqrt(cs18 Ptotal + tau2)/2, omega_eff = 1/tau; the returned
// moments carry K = omega_eff scale w per weight class, so pair16 / rest16
// with om1 = 1 - omega_eff give the relaxation. Oracle: fast16_les_cell.
__device__ __forceinline__ Mom16 moments16_les(const float (&y)[Q], const StepK& k, float& om1) {
  const float sp = __fadd_rn(__fadd_rn(__fadd_rn(y[0], y[1]), __fadd_rn(y[2], y[3])), y[4]);
  const float sm = __fadd_rn(__fadd_rn(__fadd_rn(y[9], y[10]), __fadd_rn(y[11], y[12])), y[13]);
  const float s0 = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(y[5], y[6]), __fadd_rn(y[7], y[8])),
                                       __fadd_rn(__fadd_rn(y[14], y[15]), __fadd_rn(y[16], y[17]))),
                             y[18]);
  const float sum = __fadd_rn(__fadd_rn(sp, sm), s0);
  const float jx = __fsub_rn(sp, sm);
  const float jyp = __fadd_rn(__fadd_rn(__fadd_rn(y[2], y[6]), __fadd_rn(y[7], y[8])), y[11]);
  const float jym = __fadd_rn(__fadd_rn(__fadd_rn(y[0], y[9]), __fadd_rn(y[15], y[16])), y[17]);
  const float jzp = __fadd_rn(__fadd_rn(__fadd_rn(y[3], y[5]), __fadd_rn(y[6], y[12])), y[17]);
  const float jzm = __fadd_rn(__fadd_rn(__fadd_rn(y[1], y[8]), __fadd_rn(y[10], y[14])), y[15]);
  Mom16 m;
  const float dr = __fmul_rn(sum, k.inv);
  m.dr = dr;
  const float rp = __fadd_rn(1.0f, dr);
  const float r = __fmul_rn(k.inv, __frcp_rn(rp));  // = inv/(1 + dr), inv a power of two
  m.ux = __fmul_rn(jx, r);
  m.uy = __fmul_rn(__fsub_rn(jyp, jym), r);
  m.uz = __fmul_rn(__fsub_rn(jzp, jzm), r);
  const float usq = __fmaf_rn(m.uz, m.uz, __fmaf_rn(m.uy, m.uy, __fmul_rn(m.ux, m.ux)));
  m.a = __fmul_rn(-1.5f, usq);
  const float d3 = __fmul_rn(dr, 1.0f / 3.0f);
  const float rux = __fmul_rn(rp, m.ux), ruy = __fmul_rn(rp, m.uy);
  const float Pxx = __fmaf_rn(__fadd_rn(sp, sm), k.inv, -__fmaf_rn(rux, m.ux, d3));
  const float Pyy = __fmaf_rn(__fadd_rn(jyp, jym), k.inv, -__fmaf_rn(ruy, m.uy, d3));
  const float Pzz = __fmaf_rn(__fadd_rn(jzp, jzm), k.inv, -__fmaf_rn(__fmul_rn(rp, m.uz), m.uz, d3));
  const float Pxy = __fmaf_rn(__fsub_rn(__fadd_rn(y[2], y[9]), __fadd_rn(y[0], y[11])), k.inv, -__fmul_rn(rux, m.uy));
  const float Pxz = __fmaf_rn(__fsub_rn(__fadd_rn(y[3], y[10]), __fadd_rn(y[1], y[12])), k.inv, -__fmul_rn(rux, m.uz));
  const float Pyz = __fmaf_rn(__fsub_rn(__fadd_rn(y[6], y[15]), __fadd_rn(y[8], y[17])), k.inv, -__fmul_rn(ruy, m.uz));
  float pt = __fmul_rn(Pxx, Pxx);
  pt = __fmaf_rn(Pyy, Pyy, pt);
  pt = __fmaf_rn(Pzz, Pzz, pt);
  pt = __fmaf_rn(2.0f * Pxy, Pxy, pt);
  pt = __fmaf_rn(2.0f * Pxz, Pxz, pt);
  pt = __fmaf_rn(2.0f * Pyz, Pyz, pt);
  const float tau = __fadd_rn(k.tauh_f, __fmul_rn(0.5f, __fsqrt_rn(__fmaf_rn(k.cs18_f, __fsqrt_rn(pt), k.tau2_f))));
  const float om = __frcp_rn(tau);  // = 1/tau rounded once, as a division would
  om1 = __fsub_rn(1.0f, om);
  const float oms = __fmul_rn(om, k.scale);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float K = __fmul_rn(oms, c == 0 ? 1.0f / 3.0f : (c == 1 ? 1.0f / 18.0f : 1.0f / 36.0f));
    const float kd = __fmul_rn(K, dr);
    const float kr = __fadd_rn(K, kd);
    m.kr3[c] = __fmul_rn(3.0f, kr);
    m.kr45[c] = __fmul_rn(4.5f, kr);
    m.kra[c] = __fmaf_rn(kr, m.a, kd);
  }
  return m;
}

__device__ __forceinline__ void cell16_les(const float (&y)[Q], __half (&s)[Q], const StepK& k) {
  float om1;
  const Mom16 m = moments16_les(y, k, om1);
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    float a, b;
    pair16(q, y[q], y[oppq(q)], m, om1, a, b);
    s[q] = __float2half_rn(a);
    s[oppq(q)] = __float2half_rn(b);
  }
  s[Q - 1] = __float2half_rn(rest16(y[Q - 1], m, om1));
}

struct F16 {
  using S = __half; using R = float; using V = Ex<float>;
  static constexpr int id = 2;
  // inv and scale are exact powers of two: the multiply only moves the exponent
  __device__ static __forceinline__ R dec(S s, R inv) { return __fmul_rn(__half2float(s), inv); }
  __device__ static __forceinline__ S enc(R r, R scale) { return __float2half_rn(__fmul_rn(r, scale)); }
  template <bool LES = false>
  __device__ static __forceinline__ void cell(S (&s)[Q], const StepK& k) {
    float y[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) y[q] = __half2float(s[q]);
    if constexpr (LES) {
      cell16_les(y, s, k);
      return;
    }
    const Mom16 m = moments16(y, k);
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      float a, b;
      pair16(q, y[q], y[oppq(q)], m, k.om1, a, b);
      s[q] = __float2half_rn(a);
      s[oppq(q)] = __float2half_rn(b);
    }
    s[Q - 1] = __float2half_rn(rest16(y[Q - 1], m, k.om1));
  }
};

// ----------------------------------------------------------------- geometry
// Population q of a lattice is a dense nx*ny*nz block (rows padded to sx
// elements) starting at base + q*qs. Cell (i,j,k) is at i + sx*(j + ny*k).
struct Geo {
  int nx, ny, nz;
  int sx;          // row pitch, elements (multiple of 32)
  long long qs;    // population stride, elements
  int z0 = 0;      // z-slab: global index of local plane 0 (0 for a whole box)
  int gz = 0;      // z-slab: global box height (nz for a whole box)
};

// Ghost planes of a z-slab. The plane below the slab (z = -1) holds the five
// cz = +1 populations, the plane above (z = nz) the five cz = -1 ones, each a
// sx*ny plane indexed i + sx*j. `in` are this slab's ghost planes for the
// current step; `up` / `dn` are the neighbours' planes (above: its lower plane;
// below: its upper plane) that this step's boundary planes fill for the next.
template <class S> struct Halo {
  const S* in_lo[NZF];
  const S* in_hi[NZF];
  S* up[NZF];
  S* dn[NZF];
};

template <class S> struct Pops { S* p[Q]; };

// --------------------------------------------------------- per-cell physics
// Moments and equilibrium deviation in the reference's evaluation order
// (SRC/col_MC.F90:133-219). x: pulled deviations; e: equilibrium deviations.
template <class V>
__device__ __forceinline__ V equilibrium(const V (&x)[Q], V (&e)[Q], V& vxo, V& vyo, V& vzo) {
  using N = Num<V>;
  const V uno = N::c(1.0), cte1 = N::c(1.0), cte0 = uno - cte1;
  const V rf = N::c(3.0), qf = N::c(1.5), tre = N::c(3.0);
  const V p0 = N::c(1.0 / 3.0), p1 = N::c(1.0 / 18.0), p2 = N::c(1.0 / (3.0 * 3.0 * (1.0 + 3.0)));
  V rho = x[0] + x[1] + x[2] + x[3] + x[4] + x[5] + x[6] + x[7]
        + x[8] + x[9] + x[10] + x[11] + x[12] + x[13] + x[14] + x[15]
        + x[16] + x[17] + x[18] + cte1;
  V rhoinv = uno / rho;
  V vx = (x[0] + x[1] + x[2] + x[3] + x[4] - x[9] - x[10] - x[11] - x[12] - x[13]) * rhoinv;
  V vy = (x[2] + x[6] + x[7] + x[8] + x[11] - x[0] - x[9] - x[15] - x[16] - x[17]) * rhoinv;
  V vz = (x[3] + x[5] + x[6] + x[12] + x[17] - x[1] - x[8] - x[10] - x[14] - x[15]) * rhoinv;
  vxo = vx; vyo = vy; vzo = vz;
  V vx2 = vx * vx, vy2 = vy * vy, vz2 = vz * vz;
  V vsq = vx2 + vy2 + vz2;
  V vxpy = vx + vy; V qxpy = cte0 + qf * (tre * vxpy * vxpy - vsq);
  V vxmy = vx - vy; V qxmy = cte0 + qf * (tre * vxmy * vxmy - vsq);
  V vxpz = vx + vz; V qxpz = cte0 + qf * (tre * vxpz * vxpz - vsq);
  V vxmz = vx - vz; V qxmz = cte0 + qf * (tre * vxmz * vxmz - vsq);
  V vypz = vy + vz; V qypz = cte0 + qf * (tre * vypz * vypz - vsq);
  V vymz = vy - vz; V qymz = cte0 + qf * (tre * vymz * vymz - vsq);
  V qx = cte0 + qf * (tre * vx2 - vsq);
  V qy = cte0 + qf * (tre * vy2 - vsq);
  V qz = cte0 + qf * (tre * vz2 - vsq);
  V q0 = cte0 + qf * (-vsq);
  vx = rf * vx; vy = rf * vy; vz = rf * vz;
  vxpy = rf * vxpy; vxmy = rf * vxmy; vxpz = rf * vxpz;
  vxmz = rf * vxmz; vypz = rf * vypz; vymz = rf * vymz;
  V rp0 = rho * p0, rp1 = rho * p1, rp2 = rho * p2;
  V s2 = cte1 * (rp2 - p2), s1 = cte1 * (rp1 - p1), s0 = cte1 * (rp0 - p0);
  e[0]  = rp2 * (vxmy + qxmy) + s2;
  e[1]  = rp2 * (vxmz + qxmz) + s2;
  e[2]  = rp2 * (vxpy + qxpy) + s2;
  e[3]  = rp2 * (vxpz + qxpz) + s2;
  e[4]  = rp1 * (vx + qx) + s1;
  e[5]  = rp1 * (vz + qz) + s1;
  e[6]  = rp2 * (vypz + qypz) + s2;
  e[7]  = rp1 * (vy + qy) + s1;
  e[8]  = rp2 * (vymz + qymz) + s2;
  e[9]  = rp2 * (-vxpy + qxpy) + s2;
  e[10] = rp2 * (-vxpz + qxpz) + s2;
  e[11] = rp2 * (-vxmy + qxmy) + s2;
  e[12] = rp2 * (-vxmz + qxmz) + s2;
  e[13] = rp1 * (-vx + qx) + s1;
  e[14] = rp1 * (-vz + qz) + s1;
  e[15] = rp2 * (-vypz + qypz) + s2;
  e[16] = rp1 * (-vy + qy) + s1;
  e[17] = rp2 * (-vymz + qymz) + s2;
  e[18] = rp0 * q0 + s0;
  return rho;
}

// BGK relaxation x <- x - omega*(x - e) (SRC/col_MC.F90:333-351), in place.
template <class V>
__device__ __forceinline__ void collide(V (&x)[Q], V omega) {
  V e[Q], vx, vy, vz;
  (void)equilibrium<V>(x, e, vx, vy, vz);
#pragma unroll
  for (int q = 0; q < Q; ++q) x[q] = x[q] - omega * (x[q] - e[q]);
}

template <class V>
__device__ __forceinline__ V ptotal(const V (&x)[Q], const V (&e)[Q]);

// Smagorinsky relaxation of the reference's LES block (SRC/col_MC.F90:221-309,
// disabled there by a stop): Ptotal = sqrt(Pi_neq:Pi_neq),
// Ts = 1/(2 omega1) + sqrt(18 cteS^2 Ptotal + (1/omega1)^2)/2, omega = 1/Ts,
// then the BGK update with that omega.
template <class V>
__device__ __forceinline__ void collide_les(V (&x)[Q], V cs18, V tauh, V tau2) {
  using N = Num<V>;
  V e[Q], vx, vy, vz;
  (void)equilibrium<V>(x, e, vx, vy, vz);
  const V pt = esqrt(ptotal<V>(x, e));
  const V ts = tauh + esqrt(cs18 * pt + tau2) / N::c(2.0);
  const V omega = N::c(1.0) / ts;
#pragma unroll
  for (int q = 0; q < Q; ++q) x[q] = x[q] - omega * (x[q] - e[q]);
}

// Ptotal = Pi_neq : Pi_neq with doubled off-diagonals (SRC/dissipation.F90:171-247).
template <class V>
__device__ __forceinline__ V ptotal(const V (&x)[Q], const V (&e)[Q]) {
  using N = Num<V>;
  V n[18];
#pragma unroll
  for (int q = 0; q < 18; ++q) n[q] = x[q] - e[q];
  V Pxx = n[0] + n[1] + n[2] + n[3] + n[4] + n[9] + n[10] + n[11] + n[12] + n[13];
  V Pyy = n[0] + n[2] + n[6] + n[7] + n[8] + n[9] + n[11] + n[15] + n[16] + n[17];
  V Pzz = n[1] + n[3] + n[5] + n[6] + n[8] + n[10] + n[12] + n[14] + n[15] + n[17];
  V Pxz = -n[1] + n[3] + n[10] - n[12];
  V Pxy = -n[0] + n[2] + n[9] - n[11];
  V Pyz = n[6] - n[8] + n[15] - n[17];
  const V two = N::c(2.0);
  return (Pxx * Pxx) + (Pyy * Pyy) + (Pzz * Pzz) + (two * Pxy * Pxy) + (two * Pxz * Pxz) + (two * Pyz * Pyz);
}

}  // namespace bgk
