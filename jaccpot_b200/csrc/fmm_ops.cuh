// Device-side real-basis (Dehnen, no-sqrt2) expansion algebra, fully unrolled
// for a compile-time order P so that coefficient vectors live in registers and
// the B_U entries become constant-bank operands of the FMAs.
//
// Conventions restate jaccpot/operators:
//   U_n^m(d) = r^n P_n^|m|(cos t) {cos,sin}(|m| phi) / (n+|m|)!      (real_p2m_l2p.py:51-232)
//   packed index n^2 + n + m                                          (_sh_indexing.py:36-118)
//   rotate-to-z (multipole) = B_U Dz(-ax) B_U Dz(az), az = atan2(x,y), ax = atan2(rho,z)
//                                                                     (real_rotations.py:340-503)
//   local rotations are the transposes                                (real_rotations.py:541-649)
//   z-M2L  F_n^m = sum_{k=|m|}^{p-n} sgn(m) (n+k)! r^-(n+k+1) M_k^m,  sgn = (-1)^m (2 if m!=0)
//   z-M2M  M'_n^m = sum_{k=0}^{n-|m|} dz^k/k! M_{n-k}^m
//   z-L2L  F'_n^m = sum_{k=0}^{p-n}   dz^k/k! F_{n+k}^m               (real_translations.py:72-335)
//
// Numerical form (same mathematics, different evaluation):
//   * U_n^m comes from the Cartesian recurrence of R_n^m = U_n^m + i U_n^-m,
//       R_m^m = R_{m-1}^{m-1} (x+iy)/(2m),  R_{m+1}^m = z R_m^m,
//       R_n^m = ((2n-1) z R_{n-1}^m - r^2 R_{n-2}^m) / (n^2 - m^2),
//     instead of Legendre-in-cos(theta) times Chebyshev-in-phi (no rho/r divisions);
//   * the L2P gradient uses the ladder relations  dR_n^m/dz = R_{n-1}^m,
//     (d/dx - i d/dy) R_n^m = R_{n-1}^{m-1}, (d/dx + i d/dy) R_n^m = -R_{n-1}^{m+1}
//     (the half-integer transverse identities of the reference's
//     test_solid_harmonic_transverse_derivative_coefficients_are_half_integers)
//     instead of autodiff through the recurrence;
//   * the z-M2L is evaluated in scaled form, M_k r^-k and F_n r^(n+1), which
//     avoids the r^-(n+k+1) overflow of the literal formula in float32;
//   * cos(m a), sin(m a) come from angle addition on (cos a, sin a) read off
//     the displacement, not from atan2 + cos/sin.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "generated/bu_tables.h"
#include "generated/kfold_tables.h"
#include "generated/bu_code.h"

namespace jb {

__host__ __device__ constexpr int csize(int p) { return (p + 1) * (p + 1); }
__host__ __device__ constexpr int cstride(int p) { return (csize(p) + 3) & ~3; }
__host__ __device__ constexpr int shi(int n, int m) { return n * n + n + m; }
__host__ __device__ constexpr int iabs(int a) { return a < 0 ? -a : a; }
// sum_{k<l} (2k+1)^2
__host__ __device__ constexpr int bu_off(int l) { return l * (4 * l * l - 1) / 3; }
// Sparsity of B_U (checked against the table when it is generated).
__host__ __device__ constexpr bool bu_nz(int l, int i, int j) {
  return ((i - l >= 0) != (j - l >= 0))
             ? false
             : ((i - l >= 0) ? (((l + (i - l) + (j - l)) & 1) == 0)
                             : (((l + iabs(i - l) + iabs(j - l)) & 1) == 1));
}
__host__ __device__ constexpr double factd(int n) { return n <= 1 ? 1.0 : (double)n * factd(n - 1); }

// cos(m a), sin(m a) for m = 0..P by angle addition.
template <int P>
struct Trig {
  float c[P + 1], s[P + 1];
  __device__ __forceinline__ void init(float c1, float s1) {
    c[0] = 1.f;
    s[0] = 0.f;
#pragma unroll
    for (int m = 1; m <= P; ++m) {
      c[m] = c[m - 1] * c1 - s[m - 1] * s1;
      s[m] = s[m - 1] * c1 + c[m - 1] * s1;
    }
  }
};

// v <- Dz(sign * a) v on every degree (real_rotations.py:75-147).
template <int P, bool NEG>
__device__ __forceinline__ void dz_apply(float* v, const Trig<P>& t) {
#pragma unroll
  for (int l = 1; l <= P; ++l) {
#pragma unroll
    for (int m = 1; m <= l; ++m) {
      const float c = t.c[m];
      const float s = NEG ? -t.s[m] : t.s[m];
      const int ip = shi(l, m), im = shi(l, -m);
      const float vp = v[ip], vm = v[im];
      v[ip] = c * vp - s * vm;
      v[im] = fmaf(s, vp, c * vm);
    }
  }
}

// v <- B v (TR = false) or B^T v (TR = true) per degree.  LIM_OUT: only rows
// with |m| <= P - l are produced (the rest are set to 0); LIM_IN: columns with
// |m| > P - l are known to be zero and skipped.
template <int P, bool TR, bool LIM_OUT, bool LIM_IN>
__device__ __forceinline__ void bu_apply(float* v) {
#pragma unroll
  for (int l = 1; l <= P; ++l) {
    constexpr int W = 2 * P + 1;
    const int w = 2 * l + 1, o = l * l;
    float out[W];
#pragma unroll
    for (int i = 0; i < w; ++i) {
      const int mi = i - l;
      float acc = 0.f;
      if (!(LIM_OUT && iabs(mi) > P - l)) {
#pragma unroll
        for (int j = 0; j < w; ++j) {
          const int mj = j - l;
          if (LIM_IN && iabs(mj) > P - l) continue;
          if (TR ? !bu_nz(l, j, i) : !bu_nz(l, i, j)) continue;
          const float b = TR ? c_BU[bu_off(l) + j * w + i] : c_BU[bu_off(l) + i * w + j];
          acc = fmaf(b, v[o + j], acc);
        }
      }
      out[i] = acc;
    }
#pragma unroll
    for (int i = 0; i < w; ++i) v[o + i] = out[i];
  }
}

// Rotation angles of the displacement d (alignment_angles, real_rotations.py:340-415):
// az = atan2(x, y) -> (cos, sin) = (y/rho, x/rho);  ax = atan2(rho, z) -> (z/r, rho/r).
template <int P>
__device__ __forceinline__ void align_trig(float x, float y, float z, Trig<P>& taz, Trig<P>& tax, float* r_out) {
  const float rho2 = x * x + y * y;
  const float r2 = rho2 + z * z;
  float caz = 1.f, saz = 0.f, cax = 1.f, sax = 0.f;
  const float rho = sqrtf(rho2);
  const float r = sqrtf(r2);
  if (rho2 > 0.f) {
    const float ir = 1.f / rho;
    caz = y * ir;
    saz = x * ir;
  }
  if (r2 > 0.f) {
    const float ir = 1.f / r;
    cax = z * ir;
    sax = rho * ir;
  }
  taz.init(caz, saz);
  tax.init(cax, sax);
  *r_out = r;
}

template <int P>
__device__ __forceinline__ void rot_mult_to_z(float* v, const Trig<P>& taz, const Trig<P>& tax, bool lim_out_only_for_m2l) {
  (void)lim_out_only_for_m2l;
  dz_apply<P, false>(v, taz);
  bu_apply<P, false, false, false>(v);
  dz_apply<P, true>(v, tax);
  bu_apply<P, false, false, false>(v);
}

// 1/sqrt(x) by the PTX instruction rsqrt.approx.ftz.f32 (the approximate
// reciprocal square root with subnormal inputs and results flushed to zero).
// For squared distances in the normal FP32 range its results equal rsqrtf()'s
// bit for bit (tests/test_gpu_leaf_form.py compares the two forms).  A squared
// distance below 2^-126 (points closer than about 1e-19) reads as 0 here
// (infinite 1/r, as for coincident points).
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// acc += wt * Dz(+a) v (NEG = false) or wt * Dz(-a) v (NEG = true): dz_rot's
// rotation with each rotated pair added into acc by two FMAs (no separate
// add); W = false takes wt = 1 (and W = true with wt = 1 gives the same bits).
template <int P, bool NEG, bool W = false>
__device__ __forceinline__ void dz_rot_acc(const float* v, float* acc, float c1, float s1, float wt = 1.f) {
#pragma unroll
  for (int l = 0; l <= P; ++l) acc[shi(l, 0)] = W ? fmaf(wt, v[shi(l, 0)], acc[shi(l, 0)]) : acc[shi(l, 0)] + v[shi(l, 0)];
  const float sa = NEG ? -s1 : s1;
  float c = c1, s = sa;
#pragma unroll
  for (int m = 1; m <= P; ++m) {
    if (m > 1) {
      const float cn = c * c1 - s * sa;
      s = fmaf(s, c1, c * sa);
      c = cn;
    }
    const float cw = W ? c * wt : c, sw = W ? s * wt : s;
#pragma unroll
    for (int l = m; l <= P; ++l) {
      const int ip = shi(l, m), im = shi(l, -m);
      const float vp = v[ip], vm = v[im];
      acc[ip] = fmaf(cw, vp, fmaf(-sw, vm, acc[ip]));
      acc[im] = fmaf(sw, vp, fmaf(cw, vm, acc[im]));
    }
  }
}

// v <- Dz(+a) v (NEG = false) or Dz(-a) v (NEG = true) on every degree, with
// (cos a, sin a) = (c1, s1); cos/sin(m a) by angle addition, m outermost so
// that only four trig values are live.
template <int P, bool NEG>
__device__ __forceinline__ void dz_rot(float* v, float c1, float s1) {
  const float sa = NEG ? -s1 : s1;
  float c = c1, s = sa;
#pragma unroll
  for (int m = 1; m <= P; ++m) {
    if (m > 1) {
      const float cn = c * c1 - s * sa;
      s = fmaf(s, c1, c * sa);
      c = cn;
    }
#pragma unroll
    for (int l = m; l <= P; ++l) {
      const int ip = shi(l, m), im = shi(l, -m);
      const float vp = v[ip], vm = v[im];
      v[ip] = c * vp - s * vm;
      v[im] = fmaf(s, vp, c * vm);
    }
  }
}

// v[degree n] *= s^(n + OFF) for n = 0..P.
template <int P, int OFF>
__device__ __forceinline__ void scale_degrees(float* v, float s) {
  float f = 1.f;
#pragma unroll
  for (int k = 0; k < OFF; ++k) f *= s;
#pragma unroll
  for (int n = 0; n <= P; ++n) {
#pragma unroll
    for (int m = -n; m <= n; ++m) v[shi(n, m)] *= f;
    f *= s;
  }
}

// z-axis M2L in scaled form (defined below).
template <int P>
__device__ __forceinline__ void zm2l(float* Mz, float* Lz, float r);

// One M2L in place, delta = target - source, as the chain
//   Dz(az) -> B -> Dz(-ax) -> r^-k -> K -> r^-(n+1) -> Dz(ax) -> B^T -> Dz(-az)
// which is the reference's rotate-to-z / z-M2L / rotate-back cascade
// (operators/m2l_real_rot_scale.py:288-386) with its middle B^T Z B folded
// into the constant K (B commutes with the per-degree radius scalings).
template <int P>
__device__ __forceinline__ void m2l_kfold(float* v, float dx, float dy, float dz) {
  const float rho2 = dx * dx + dy * dy;
  const float r2 = rho2 + dz * dz;
  float caz = 1.f, saz = 0.f, cax = 1.f, sax = 0.f;
  const float rho = sqrtf(rho2);
  const float r = sqrtf(r2);
  if (rho2 > 0.f) {
    const float ir = 1.f / rho;
    caz = dy * ir;
    saz = dx * ir;
  }
  if (r2 > 0.f) {
    const float ir = 1.f / r;
    cax = dz * ir;
    sax = rho * ir;
  }
  const float s = 1.f / fmaxf(r, 1.0e-30f);
  if constexpr (P <= 8) {
    dz_rot<P, false>(v, caz, saz);
    BApply<P, false>::apply(v);
    dz_rot<P, true>(v, cax, sax);
    scale_degrees<P, 0>(v, s);
    KFold<P>::apply(v);
    scale_degrees<P, 1>(v, s);
    dz_rot<P, false>(v, cax, sax);
    BApply<P, true>::apply(v);
    dz_rot<P, true>(v, caz, saz);
  } else {
    // From order 9 the entries of K are no longer exact in FP32 and the
    // folded product loses the cancellations that the factored form keeps,
    // so the three constant factors are applied one after the other.
    dz_rot<P, false>(v, caz, saz);
    BApply<P, false>::apply(v);
    dz_rot<P, true>(v, cax, sax);
    BApply<P, false>::apply(v);
    float w[csize(P)];
    zm2l<P>(v, w, r);
    BApply<P, true>::apply(w);
    dz_rot<P, false>(w, cax, sax);
    BApply<P, true>::apply(w);
    dz_rot<P, true>(w, caz, saz);
#pragma unroll
    for (int k = 0; k < csize(P); ++k) v[k] = w[k];
  }
}

// acc += wt * M2L(d) v (v is overwritten; W = false: wt = 1): the chain of
// m2l_kfold for P <= 8 with the angles' 1/rho and 1/r from the approximate
// reciprocal square root (instead of correctly rounded square roots and
// divisions; the rotation cosines and sines move by about one ulp) and the
// last z-rotation accumulating into acc.  The thread-per-unit M2L kernel uses
// this form.
template <int P, bool W = false>
__device__ __forceinline__ void m2l_kfold_acc(float* v, float* acc, float dx, float dy, float dz, float wt = 1.f) {
  if constexpr (P <= 8) {
    const float rho2 = dx * dx + dy * dy;
    const float r2 = rho2 + dz * dz;
    float caz = 1.f, saz = 0.f, cax = 1.f, sax = 0.f, rho = 0.f, s = 1.0e30f;
    if (rho2 > 0.f) {
      const float ir = rsqrt_ftz(rho2);
      caz = dy * ir;
      saz = dx * ir;
      rho = rho2 * ir;
    }
    if (r2 > 0.f) {
      const float ir = rsqrt_ftz(r2);
      cax = dz * ir;
      sax = rho * ir;
      s = ir;
    }
    dz_rot<P, false>(v, caz, saz);
    BApply<P, false>::apply(v);
    dz_rot<P, true>(v, cax, sax);
    scale_degrees<P, 0>(v, s);
    KFold<P>::apply(v);
    scale_degrees<P, 1>(v, s);
    dz_rot<P, false>(v, cax, sax);
    BApply<P, true>::apply(v);
    dz_rot_acc<P, true, W>(v, acc, caz, saz, wt);
  } else {
    m2l_kfold<P>(v, dx, dy, dz);
#pragma unroll
    for (int k = 0; k < csize(P); ++k) acc[k] = W ? fmaf(wt, v[k], acc[k]) : acc[k] + v[k];
  }
}

// z-M2L in scaled form; Mz is the rotated multipole, Lz the z-frame local.
template <int P>
__device__ __forceinline__ void zm2l(float* Mz, float* Lz, float r) {
  const float s = 1.f / fmaxf(r, 1.0e-30f);
  float sp[P + 2];
  sp[0] = 1.f;
#pragma unroll
  for (int k = 1; k <= P + 1; ++k) sp[k] = sp[k - 1] * s;
#pragma unroll
  for (int k = 1; k <= P; ++k) {
#pragma unroll
    for (int m = -k; m <= k; ++m) Mz[shi(k, m)] *= sp[k];
  }
#pragma unroll
  for (int n = 0; n <= P; ++n) {
#pragma unroll
    for (int m = -n; m <= n; ++m) {
      const int am = iabs(m);
      float acc = 0.f;
#pragma unroll
      for (int k = am; k <= P - n; ++k) acc = fmaf((float)factd(n + k), Mz[shi(k, m)], acc);
      const float sg = ((am & 1) ? -1.f : 1.f) * (m != 0 ? 2.f : 1.f);
      Lz[shi(n, m)] = (am > P - n) ? 0.f : sg * sp[n + 1] * acc;
    }
  }
}

// One M2L: out = from_z_local( zm2l( to_z_mult(M) ) ), delta = target - source.
template <int P>
__device__ __forceinline__ void m2l_pair(float* v, float* w, float dx, float dy, float dz) {
  Trig<P> taz, tax;
  float r;
  align_trig<P>(dx, dy, dz, taz, tax, &r);
  // to-z multipole: B Dz(-ax) B Dz(az); only rows |m| <= P-l of the last B are used.
  dz_apply<P, false>(v, taz);
  bu_apply<P, false, false, false>(v);
  dz_apply<P, true>(v, tax);
  bu_apply<P, false, true, false>(v);
  zm2l<P>(v, w, r);
  // from-z local: Dz(-az) B^T Dz(ax) B^T; the z-frame local is zero for |m| > P-l.
  bu_apply<P, true, false, true>(w);
  dz_apply<P, false>(w, tax);
  bu_apply<P, true, false, false>(w);
  dz_apply<P, true>(w, taz);
}

// Rotation angles of a displacement as (cos, sin) pairs for dz_rot:
// az = atan2(x, y) -> (y/rho, x/rho);  ax = atan2(rho, z) -> (z/r, rho/r).
__device__ __forceinline__ void align_cs(float x, float y, float z, float& caz, float& saz, float& cax, float& sax,
                                         float& r) {
  const float rho2 = x * x + y * y;
  const float r2 = rho2 + z * z;
  const float rho = sqrtf(rho2);
  r = sqrtf(r2);
  caz = 1.f;
  saz = 0.f;
  cax = 1.f;
  sax = 0.f;
  if (rho2 > 0.f) {
    const float ir = 1.f / rho;
    caz = y * ir;
    saz = x * ir;
  }
  if (r2 > 0.f) {
    const float ir = 1.f / r;
    cax = z * ir;
    sax = rho * ir;
  }
}

// M2M: delta = child - parent (source - destination).  r < 1e-30 -> identity shift.
template <int P>
__device__ __forceinline__ void m2m_pair(float* v, float dx, float dy, float dz) {
  float caz, saz, cax, sax, r;
  align_cs(dx, dy, dz, caz, saz, cax, sax, r);
  const float d = r < 1e-30f ? 0.f : r;
  dz_rot<P, false>(v, caz, saz);
  BApply<P, false>::apply(v);
  dz_rot<P, true>(v, cax, sax);
  BApply<P, false>::apply(v);
  float dk[P + 1];
  dk[0] = 1.f;
#pragma unroll
  for (int k = 1; k <= P; ++k) dk[k] = dk[k - 1] * d * (float)(1.0 / (double)k);
  // in place, highest degree first (sources are lower degrees)
#pragma unroll
  for (int n = P; n >= 1; --n) {
#pragma unroll
    for (int m = -n; m <= n; ++m) {
      float acc = v[shi(n, m)];
#pragma unroll
      for (int k = 1; k <= n - iabs(m); ++k) acc = fmaf(dk[k], v[shi(n - k, m)], acc);
      v[shi(n, m)] = acc;
    }
  }
  // from-z multipole: Dz(-az) B Dz(ax) B
  BApply<P, false>::apply(v);
  dz_rot<P, false>(v, cax, sax);
  BApply<P, false>::apply(v);
  dz_rot<P, true>(v, caz, saz);
}

// L2L: delta = parent - child (old - new centre).
template <int P>
__device__ __forceinline__ void l2l_pair(float* v, float dx, float dy, float dz) {
  float caz, saz, cax, sax, r;
  align_cs(dx, dy, dz, caz, saz, cax, sax, r);
  const float d = r < 1e-30f ? 0.f : r;
  // to-z local: B^T Dz(-ax) B^T Dz(az)
  dz_rot<P, false>(v, caz, saz);
  BApply<P, true>::apply(v);
  dz_rot<P, true>(v, cax, sax);
  BApply<P, true>::apply(v);
  float dk[P + 1];
  dk[0] = 1.f;
#pragma unroll
  for (int k = 1; k <= P; ++k) dk[k] = dk[k - 1] * d * (float)(1.0 / (double)k);
  // in place, lowest degree first (sources are higher degrees)
#pragma unroll
  for (int n = 0; n < P; ++n) {
#pragma unroll
    for (int m = -n; m <= n; ++m) {
      float acc = v[shi(n, m)];
#pragma unroll
      for (int k = 1; k <= P - n; ++k) acc = fmaf(dk[k], v[shi(n + k, m)], acc);
      v[shi(n, m)] = acc;
    }
  }
  // from-z local: Dz(-az) B^T Dz(ax) B^T
  BApply<P, true>::apply(v);
  dz_rot<P, false>(v, cax, sax);
  BApply<P, true>::apply(v);
  dz_rot<P, true>(v, caz, saz);
}

// U_n^m(d) for all n <= P.
template <int P>
__device__ __forceinline__ void solid_harmonics(float x, float y, float z, float* U) {
  const float r2 = x * x + y * y + z * z;
  float re = 1.f, im = 0.f;  // R_m^m
#pragma unroll
  for (int m = 0; m <= P; ++m) {
    if (m > 0) {
      const float f = 0.5f / (float)m;
      const float nr = (re * x - im * y) * f;
      const float ni = (re * y + im * x) * f;
      re = nr;
      im = ni;
    }
    U[shi(m, m)] = re;
    if (m > 0) U[shi(m, -m)] = im;
    if (m + 1 <= P) {
      U[shi(m + 1, m)] = z * re;
      if (m > 0) U[shi(m + 1, -m)] = z * im;
    }
#pragma unroll
    for (int n = m + 2; n <= P; ++n) {
      const float a = (float)(2 * n - 1);
      const float inv = (float)(1.0 / (double)((n - m) * (n + m)));
      U[shi(n, m)] = (a * z * U[shi(n - 1, m)] - r2 * U[shi(n - 2, m)]) * inv;
      if (m > 0) U[shi(n, -m)] = (a * z * U[shi(n - 1, -m)] - r2 * U[shi(n - 2, -m)]) * inv;
    }
  }
}

// Potential and gradient (w.r.t. delta) of sum F U(delta); F read through Fp.
template <int P, typename FP>
__device__ __forceinline__ void l2p_eval(const FP& F, const float* U, float* phi, float* g) {
  float p0 = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
#pragma unroll
  for (int n = 0; n <= P; ++n) {
#pragma unroll
    for (int m = -n; m <= n; ++m) p0 = fmaf(F(shi(n, m)), U[shi(n, m)], p0);
  }
  // U_{q}^{mm} for degree q = n-1, with the conventions U^{-0} = 0 and 0 outside |mm| <= q.
#define JB_UL(q, mm) ((iabs(mm) > (q)) ? 0.f : (((mm) == 0 && false) ? 0.f : U[shi((q), (mm))]))
#pragma unroll
  for (int n = 1; n <= P; ++n) {
    const int q = n - 1;
    // m = 0
    {
      const float f = F(shi(n, 0));
      if (q >= 0) gz = fmaf(f, U[shi(q, 0)], gz);
      if (q >= 1) {
        gx = fmaf(-f, U[shi(q, 1)], gx);
        gy = fmaf(-f, U[shi(q, -1)], gy);
      }
    }
#pragma unroll
    for (int m = 1; m <= n; ++m) {
      const float fc = F(shi(n, m));
      const float fs = F(shi(n, -m));
      if (m <= q) {
        gz = fmaf(fc, U[shi(q, m)], gz);
        gz = fmaf(fs, U[shi(q, -m)], gz);
      }
      // cos channel
      const float up1 = (m + 1 <= q) ? U[shi(q, m + 1)] : 0.f;
      const float um1 = (m - 1 <= q) ? U[shi(q, m - 1)] : 0.f;
      const float sp1 = (m + 1 <= q) ? U[shi(q, -(m + 1))] : 0.f;
      const float sm1 = (m - 1 >= 1 && m - 1 <= q) ? U[shi(q, -(m - 1))] : 0.f;
      gx = fmaf(fc, 0.5f * (um1 - up1), gx);
      gy = fmaf(fc, -0.5f * (sp1 + sm1), gy);
      // sin channel
      gx = fmaf(fs, 0.5f * (sm1 - sp1), gx);
      gy = fmaf(fs, 0.5f * (up1 + um1), gy);
    }
  }
#undef JB_UL
  *phi = p0;
  g[0] = gx;
  g[1] = gy;
  g[2] = gz;
}

// Calls f(axis, row, col, value) for every entry of the derivative ladders
// D_a (a = x, y, z = 0, 1, 2): d/ddelta_a sum_col F[col] U_col(delta) =
// sum_row (D_a F)[row] U_row(delta), (D_a F)[row] = sum value * F[col].  These
// are the relations l2p_eval uses for the gradient; the adjoint kernels use
// them for Hessian-vector products, for the derivative of a translated
// expansion with respect to its displacement, and (transposed) for the
// derivative of U itself: dU_col/ddelta_a = sum_row D_a[row][col] U_row.
template <int P, typename Fn>
__device__ __forceinline__ void for_ladder(Fn&& f) {
#pragma unroll
  for (int n = 1; n <= P; ++n) {
    const int q = n - 1;
    f(2, shi(q, 0), shi(n, 0), 1.f);
    if (q >= 1) {
      f(0, shi(q, 1), shi(n, 0), -1.f);
      f(1, shi(q, -1), shi(n, 0), -1.f);
    }
#pragma unroll
    for (int m = 1; m <= n; ++m) {
      const int fc = shi(n, m), fs = shi(n, -m);
      if (m <= q) {
        f(2, shi(q, m), fc, 1.f);
        f(2, shi(q, -m), fs, 1.f);
      }
      if (m - 1 <= q) {
        f(0, shi(q, m - 1), fc, 0.5f);
        f(1, shi(q, m - 1), fs, 0.5f);
        if (m - 1 >= 1) {
          f(1, shi(q, -(m - 1)), fc, -0.5f);
          f(0, shi(q, -(m - 1)), fs, 0.5f);
        }
      }
      if (m + 1 <= q) {
        f(0, shi(q, m + 1), fc, -0.5f);
        f(1, shi(q, -(m + 1)), fc, -0.5f);
        f(0, shi(q, -(m + 1)), fs, -0.5f);
        f(1, shi(q, m + 1), fs, 0.5f);
      }
    }
  }
}

// g[a] = sum_row X[row] (D_a F)[row] for a = x, y, z.
template <int P, typename FX, typename FF>
__device__ __forceinline__ void ladder_dot3(const FX& X, const FF& F, float* g) {
  float gx = 0.f, gy = 0.f, gz = 0.f;
  for_ladder<P>([&](int a, int row, int col, float val) {
    const float t = val * X(row) * F(col);
    if (a == 0) gx += t;
    else if (a == 1) gy += t;
    else gz += t;
  });
  g[0] = gx;
  g[1] = gy;
  g[2] = gz;
}

}  // namespace jb
