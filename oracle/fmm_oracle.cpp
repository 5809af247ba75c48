// TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.
//
// CPU restatement of jaccpot's real-basis (Dehnen, no-sqrt2) FMM evaluation pass.
// It is the checker for the CUDA kernels in jaccpot_b200/csrc and the timed CPU
// baseline ("port") in bench.py.  Only tests/, __graft_entry__.smoke() and
// bench.py's CPU legs load it.  Every routine cites the reference file:line it
// restates (paths relative to the jaccpot project root).
//
// Deliberate, documented deviations from the reference's arithmetic:
//   * factorials are exact values rounded to T; the reference tabulates
//     exp(lgamma(n+1)) in T (operators/_sh_indexing.py:120-147), which carries up
//     to 4.4e-6 relative error in float32 and 1.4e-14 in float64;
//   * rotation blocks are applied factor by factor (Dz, B, Dz, B) instead of
//     assembling the (2l+1)^2 block first (operators/real_rotations.py:417-503);
//     the product is the same matrix, only the rounding order differs.
//
// Build: oracle/Makefile -> oracle/_build/libjaccpot_oracle.so (OpenMP).

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// operators/_sh_indexing.py:36-118 — packed layout, degree n at [n^2, n^2+2n+1),
// m = -n..n at n^2 + n + m.
static inline int sh_size(int p) { return (p + 1) * (p + 1); }
static inline int sh_index(int n, int m) { return n * n + n + m; }

// operators/dtypes.py squared_radius_floor: max(1e-60, finfo(T).tiny).
template <typename T> static inline T sq_floor();
template <> inline double sq_floor<double>() { return 1e-60; }
template <> inline float sq_floor<float>() { return FLT_MIN; }

static double fact_exact(int n) {
  double f = 1.0;
  for (int i = 2; i <= n; ++i) f *= (double)i;
  return f;
}

// ---------------------------------------------------------------------------
// B matrices.  operators/real_dehnen_q.py:49-143 (complex recursion, Dehnen 2014
// eq. 63), :146-199 (Q, no sqrt2), :300-380 (B_U = Q B_complex^T Q^-1).
// ---------------------------------------------------------------------------
static std::vector<double> complex_B(int ell) {
  std::vector<double> prev(1, 1.0);
  for (int n = 0; n < ell; ++n) {
    const int nn = n + 1, w = 2 * nn + 1, wp = 2 * n + 1;
    std::vector<double> next((size_t)w * w, 0.0);
    auto get = [&](int m, int l) -> double {
      if (std::abs(m) > n || std::abs(l) > n) return 0.0;
      return prev[(size_t)(m + n) * wp + (l + n)];
    };
    for (int mt = -nn; mt <= nn; ++mt) {
      for (int lt = -nn; lt <= nn; ++lt) {
        double v = 0.0;
        if (std::abs(mt) <= n) {
          v = 0.5 * (get(mt, lt - 1) - get(mt, lt + 1));
        } else if (mt == n + 1) {
          v = 0.5 * (get(n, lt - 1) + get(n, lt + 1) + 2.0 * get(n, lt));
        } else {
          v = 0.5 * (get(-n, lt - 1) + get(-n, lt + 1) - 2.0 * get(-n, lt));
        }
        next[(size_t)(mt + nn) * w + (lt + nn)] = v;
      }
    }
    prev.swap(next);
  }
  return prev;
}

// B_U for degree ell, row-major (2l+1)^2, float64.
static std::vector<double> real_BU(int ell) {
  typedef std::complex<double> cd;
  const int w = 2 * ell + 1;
  std::vector<double> Bc = complex_B(ell);
  std::vector<cd> Q((size_t)w * w, cd(0, 0)), Qi((size_t)w * w, cd(0, 0));
  Q[(size_t)ell * w + ell] = 1.0;
  Qi[(size_t)ell * w + ell] = 1.0;
  for (int m = 1; m <= ell; ++m) {
    const double ph = (m % 2) ? -1.0 : 1.0;
    const int p_ = ell + m, n_ = ell - m;
    Q[(size_t)p_ * w + p_] = cd(0.5, 0);
    Q[(size_t)p_ * w + n_] = cd(0.5 * ph, 0);
    Q[(size_t)n_ * w + p_] = cd(0, -0.5);
    Q[(size_t)n_ * w + n_] = cd(0, 0.5 * ph);
    // analytic inverse: Theta_+ = T_+ + i T_-, Theta_- = ph (T_+ - i T_-)
    Qi[(size_t)p_ * w + p_] = cd(1, 0);
    Qi[(size_t)p_ * w + n_] = cd(0, 1);
    Qi[(size_t)n_ * w + p_] = cd(ph, 0);
    Qi[(size_t)n_ * w + n_] = cd(0, -ph);
  }
  // tmp = Bc^T Qi
  std::vector<cd> tmp((size_t)w * w, cd(0, 0));
  for (int i = 0; i < w; ++i)
    for (int j = 0; j < w; ++j) {
      cd s(0, 0);
      for (int k = 0; k < w; ++k) s += Bc[(size_t)k * w + i] * Qi[(size_t)k * w + j];
      tmp[(size_t)i * w + j] = s;
    }
  std::vector<double> out((size_t)w * w);
  for (int i = 0; i < w; ++i)
    for (int j = 0; j < w; ++j) {
      cd s(0, 0);
      for (int k = 0; k < w; ++k) s += Q[(size_t)i * w + k] * tmp[(size_t)k * w + j];
      out[(size_t)i * w + j] = s.real();
    }
  return out;
}

struct Tables {
  int p = -1;
  std::vector<std::vector<double>> BU;  // per degree
  std::vector<double> fact;             // 0..2p+1
  void ensure(int order) {
    if (order <= p) return;
    p = order;
    BU.clear();
    for (int l = 0; l <= p; ++l) BU.push_back(real_BU(l));
    fact.resize(2 * p + 2);
    for (int i = 0; i < (int)fact.size(); ++i) fact[i] = fact_exact(i);
  }
};
// Tables are built once per order at the exported entry points (outside any
// parallel region); inner routines only read them.
static Tables g_tables;
static inline Tables& tables(int) { return g_tables; }
static void ensure_tables(int p) { g_tables.ensure(p); }

// ---------------------------------------------------------------------------
// Rotations.  operators/real_rotations.py:75-147 (Dz), :340-415 (angles),
// :417-503 (to/from-z multipole), :541-649 (local = transposes).
// ---------------------------------------------------------------------------
template <typename T>
static void dz_apply(T* v, int ell, T angle) {
  for (int m = 1; m <= ell; ++m) {
    const T a = (T)m * angle;
    const T c = std::cos(a), s = std::sin(a);
    const int ip = ell + m, im = ell - m;
    const T vp = v[ip], vm = v[im];
    v[ip] = c * vp - s * vm;
    v[im] = s * vp + c * vm;
  }
}

template <typename T>
static void bu_apply(T* v, int ell, const std::vector<double>& B, bool transpose) {
  const int w = 2 * ell + 1;
  T out[64];
  for (int i = 0; i < w; ++i) {
    T s = 0;
    for (int j = 0; j < w; ++j) {
      const T b = (T)(transpose ? B[(size_t)j * w + i] : B[(size_t)i * w + j]);
      s += b * v[j];
    }
    out[i] = s;
  }
  for (int i = 0; i < w; ++i) v[i] = out[i];
}

template <typename T>
static void alignment_angles(T x, T y, T z, T* az, T* ax) {
  const T rho_sq = x * x + y * y;
  const bool rho_pos = rho_sq > 0;
  const T rho = rho_pos ? std::sqrt(rho_sq) : (T)0;
  *az = rho_pos ? std::atan2(x, y) : (T)0;  // NOTE atan2(x, y), real_rotations.py:404
  const bool r_pos = (rho_sq + z * z) > 0;
  *ax = r_pos ? std::atan2(rho, z) : (T)0;
}

enum RotKind { MULT_TO_Z, MULT_FROM_Z, LOCAL_TO_Z, LOCAL_FROM_Z };

template <typename T>
static void rotate(T* c, int p, T az, T ax, RotKind kind) {
  Tables& tb = tables(p);
  for (int l = 0; l <= p; ++l) {
    T* v = c + l * l;
    const auto& B = tb.BU[l];
    switch (kind) {
      case MULT_TO_Z:  // B Dz(-ax) B Dz(az)
        dz_apply(v, l, az); bu_apply(v, l, B, false); dz_apply(v, l, (T)-ax); bu_apply(v, l, B, false);
        break;
      case LOCAL_FROM_Z:  // (B Dz(-ax) B Dz(az))^T = Dz(-az) B^T Dz(ax) B^T
        bu_apply(v, l, B, true); dz_apply(v, l, ax); bu_apply(v, l, B, true); dz_apply(v, l, (T)-az);
        break;
      case MULT_FROM_Z:  // Dz(-az) B Dz(ax) B
        bu_apply(v, l, B, false); dz_apply(v, l, ax); bu_apply(v, l, B, false); dz_apply(v, l, (T)-az);
        break;
      case LOCAL_TO_Z:  // (Dz(-az) B Dz(ax) B)^T = B^T Dz(-ax) B^T Dz(az)
        dz_apply(v, l, az); bu_apply(v, l, B, true); dz_apply(v, l, (T)-ax); bu_apply(v, l, B, true);
        break;
    }
  }
}

// ---------------------------------------------------------------------------
// z-axis translations.  operators/real_translations.py:72-153 (M2M/L2L shift
// tables + kernel), :213-335 (M2L tables + kernel).
// ---------------------------------------------------------------------------
template <typename T>
static void zshift(const T* in, T* out, int p, T dz, bool is_m2m) {
  Tables& tb = tables(p);
  T ck[32];
  for (int k = 0; k <= p; ++k) {
    T pw = 1;
    for (int i = 0; i < k; ++i) pw *= dz;
    ck[k] = pw / (T)tb.fact[k];
  }
  for (int n = 0; n <= p; ++n)
    for (int m = -n; m <= n; ++m) {
      const int am = std::abs(m);
      T s = 0;
      for (int k = 0; k <= p; ++k) {
        const int sn = is_m2m ? n - k : n + k;
        const bool ok = is_m2m ? (sn >= am) : (sn <= p);
        if (ok) s += in[sh_index(sn, m)] * ck[k];
      }
      out[sh_index(n, m)] = s;
    }
}

template <typename T>
static void zm2l(const T* in, T* out, int p, T r) {
  Tables& tb = tables(p);
  for (int n = 0; n <= p; ++n)
    for (int m = -n; m <= n; ++m) {
      const int am = std::abs(m);
      const T sg = (T)(((am % 2) ? -1.0 : 1.0) * (m != 0 ? 2.0 : 1.0));
      T s = 0;
      for (int k = am; k <= p - n; ++k) {
        const T rp = std::pow(r, (T)(n + k + 1));
        s += sg * (T)tb.fact[n + k] / rp * in[sh_index(k, m)];
      }
      out[sh_index(n, m)] = s;
    }
}

// operators/m2l_real_rot_scale.py:288-386 (cascade; radius floored at 1e-30 in
// m2l_core_z_real :323), delta = target - source.
template <typename T>
static void m2l(const T* M, const T* d, T* out, int p) {
  const int C = sh_size(p);
  T buf[256], lz[256];
  for (int i = 0; i < C; ++i) buf[i] = M[i];
  const T r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  T r = r2 > 0 ? std::sqrt(r2) : (T)0;
  r = std::max(r, (T)1.0e-30);
  T az, ax;
  alignment_angles(d[0], d[1], d[2], &az, &ax);
  rotate(buf, p, az, ax, MULT_TO_Z);
  zm2l(buf, lz, p, r);
  rotate(lz, p, az, ax, LOCAL_FROM_Z);
  for (int i = 0; i < C; ++i) out[i] = lz[i];
}

// operators/real_translations.py:531-601, delta = source - destination (child - parent).
template <typename T>
static void m2m(const T* M, const T* d, T* out, int p) {
  const int C = sh_size(p);
  T buf[256], bz[256];
  for (int i = 0; i < C; ++i) buf[i] = M[i];
  const T r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  const T r = std::sqrt(std::max(r2, sq_floor<T>()));
  const T dz = r < (T)1e-30 ? (T)0 : r;
  T az, ax;
  alignment_angles(d[0], d[1], d[2], &az, &ax);
  rotate(buf, p, az, ax, MULT_TO_Z);
  zshift(buf, bz, p, dz, true);
  rotate(bz, p, az, ax, MULT_FROM_Z);
  for (int i = 0; i < C; ++i) out[i] = bz[i];
}

// operators/real_translations.py:604-667, delta = old - new (parent - child).
template <typename T>
static void l2l(const T* L, const T* d, T* out, int p) {
  const int C = sh_size(p);
  T buf[256], bz[256];
  for (int i = 0; i < C; ++i) buf[i] = L[i];
  const T r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  const T r = std::sqrt(std::max(r2, sq_floor<T>()));
  const T dz = r < (T)1e-30 ? (T)0 : r;
  T az, ax;
  alignment_angles(d[0], d[1], d[2], &az, &ax);
  rotate(buf, p, az, ax, LOCAL_TO_Z);
  zshift(buf, bz, p, dz, false);
  rotate(bz, p, az, ax, LOCAL_FROM_Z);
  for (int i = 0; i < C; ++i) out[i] = bz[i];
}

// ---------------------------------------------------------------------------
// Solid harmonics U_n^m.  operators/real_p2m_l2p.py:51-232 (P2M) and :241-400
// (L2P).  Written over a scalar type S so the same code runs on duals, which
// reproduces jax.value_and_grad of evaluate_local_real (:494-547).
// ---------------------------------------------------------------------------
template <typename T>
struct Dual {
  T v, d[3];
  Dual() : v(0) { d[0] = d[1] = d[2] = 0; }
  Dual(T x) : v(x) { d[0] = d[1] = d[2] = 0; }
};
template <typename T> static inline Dual<T> operator+(Dual<T> a, Dual<T> b) { Dual<T> r; r.v = a.v + b.v; for (int i = 0; i < 3; ++i) r.d[i] = a.d[i] + b.d[i]; return r; }
template <typename T> static inline Dual<T> operator-(Dual<T> a, Dual<T> b) { Dual<T> r; r.v = a.v - b.v; for (int i = 0; i < 3; ++i) r.d[i] = a.d[i] - b.d[i]; return r; }
template <typename T> static inline Dual<T> operator*(Dual<T> a, Dual<T> b) { Dual<T> r; r.v = a.v * b.v; for (int i = 0; i < 3; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i]; return r; }
template <typename T> static inline Dual<T> operator/(Dual<T> a, Dual<T> b) { Dual<T> r; r.v = a.v / b.v; for (int i = 0; i < 3; ++i) r.d[i] = (a.d[i] * b.v - a.v * b.d[i]) / (b.v * b.v); return r; }
template <typename T> static inline Dual<T> dsqrt(Dual<T> a) { Dual<T> r; r.v = std::sqrt(a.v); for (int i = 0; i < 3; ++i) r.d[i] = a.d[i] / ((T)2 * r.v); return r; }
// jnp.maximum(r2, floor): derivative passes through where r2 wins.
template <typename T> static inline Dual<T> dfloor(Dual<T> a, T f) { if (a.v >= f) return a; return Dual<T>(f); }
template <typename T> static inline T val(T a) { return a; }
template <typename T> static inline T val(Dual<T> a) { return a.v; }
template <typename T> static inline T hsqrt(T a) { return std::sqrt(a); }
template <typename T> static inline Dual<T> hsqrt(Dual<T> a) { return dsqrt(a); }
template <typename T> static inline T hfloor(T a, T f) { return std::max(a, f); }
template <typename T> static inline Dual<T> hfloor(Dual<T> a, T f) { return dfloor(a, f); }

// Fills U[C] with U_n^m(delta) following real_p2m_l2p.py:147-230 step by step.
template <typename T, typename S>
static void solid_harmonics(const S* dlt, int p, S* U) {
  Tables& tb = tables(p);
  const S x = dlt[0], y = dlt[1], z = dlt[2];
  const S r2 = x * x + y * y + z * z;
  const S r = hsqrt(hfloor(r2, sq_floor<T>()));
  const S rho = hsqrt(hfloor(x * x + y * y, sq_floor<T>()));
  const S ct = z / r, st = rho / r;
  const S cphi = x / rho, sphi = y / rho;  // _sh_indexing.py:149-195, no branch
  S cm[32], sm[32];
  cm[0] = S((T)1); sm[0] = S((T)0);
  if (p >= 1) { cm[1] = cphi; sm[1] = sphi; }
  for (int m = 2; m <= p; ++m) {
    cm[m] = S((T)2) * cphi * cm[m - 1] - cm[m - 2];
    sm[m] = S((T)2) * cphi * sm[m - 1] - sm[m - 2];
  }
  S rn = S((T)1);
  for (int n = 0; n <= p; ++n) {
    if (n > 0) rn = rn * r;
    for (int m = -n; m <= n; ++m) {
      const int am = std::abs(m);
      S Pmm;
      if (am == 0) {
        Pmm = S((T)1);
      } else {
        const T dfact = (T)tb.fact[2 * am] / ((T)std::ldexp(1.0, am) * (T)tb.fact[am]);
        S stp = S((T)1);
        for (int i = 0; i < am; ++i) stp = stp * st;
        Pmm = S(dfact) * stp;
      }
      S Pnm;
      if (am == n) {
        Pnm = Pmm;
      } else if (am + 1 == n) {
        Pnm = S((T)(2.0 * am + 1.0)) * ct * Pmm;
      } else {
        S P2 = Pmm, P1 = S((T)(2.0 * am + 1.0)) * ct * Pmm;
        for (int k = am + 2; k <= n; ++k) {
          S num = S((T)(2.0 * k - 1.0)) * ct * P1;
          num = num - S((T)(k + am - 1.0)) * P2;
          S Pk = num / S((T)(k - am));
          P2 = P1;
          P1 = Pk;
        }
        Pnm = P1;
      }
      const S denom = S((T)tb.fact[n + am]);
      U[sh_index(n, m)] = (m >= 0) ? rn * Pnm * cm[am] / denom : rn * Pnm * sm[am] / denom;
    }
  }
}

template <typename T>
static void p2m_one(const T* d, T mass, T* out, int p) {
  T U[256];
  solid_harmonics<T, T>(d, p, U);
  for (int i = 0; i < sh_size(p); ++i) out[i] = mass * U[i];
}

// L2P: potential phi = sum F U(delta) and grad_delta phi, delta = centre - x.
template <typename T>
static void l2p_one(const T* F, const T* d, int p, T* pot, T* grad) {
  Dual<T> dd[3];
  for (int i = 0; i < 3; ++i) { dd[i] = Dual<T>(d[i]); dd[i].d[i] = 1; }
  Dual<T> U[256];
  solid_harmonics<T, Dual<T>>(dd, p, U);
  Dual<T> tot((T)0);
  for (int i = 0; i < sh_size(p); ++i) tot = tot + Dual<T>(F[i]) * U[i];
  *pot = tot.v;
  grad[0] = tot.d[0]; grad[1] = tot.d[1]; grad[2] = tot.d[2];
}

// ---------------------------------------------------------------------------
// Tree-level pass.  Topology (the yggdrax artefacts, consumed unchanged):
//   node_ranges[2*n], [2*n+1]  inclusive particle span (sorted order)
//   left/right[i] for internal i in [0, num_internal) (BFS order, root = 0)
//   leaves are nodes [num_internal, num_nodes), in particle order
//   level_off[0..num_levels] offsets of each depth's internal nodes
// ---------------------------------------------------------------------------

// COM centres: yggdrax compute_tree_mass_moments, called at
// upward/real_tree_expansions.py:439; restated as in mutual/topology.py:500-516.
template <typename T>
static void com(int64_t N, const T* pos, const T* mass, int num_nodes, const int* ranges, T* out) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int n = 0; n < num_nodes; ++n) {
    T sm = 0, sx = 0, sy = 0, sz = 0;
    for (int i = ranges[2 * n]; i <= ranges[2 * n + 1]; ++i) {
      sm += mass[i];
      sx += mass[i] * pos[3 * i]; sy += mass[i] * pos[3 * i + 1]; sz += mass[i] * pos[3 * i + 2];
    }
    if (sm > 0) {
      const T inv = (T)1 / sm;
      out[3 * n] = sx * inv; out[3 * n + 1] = sy * inv; out[3 * n + 2] = sz * inv;
    } else {  // no mass: mean position (mutual/topology.py:500-516)
      T mx = 0, my = 0, mz = 0;
      const int cnt = ranges[2 * n + 1] - ranges[2 * n] + 1;
      for (int i = ranges[2 * n]; i <= ranges[2 * n + 1]; ++i) {
        mx += pos[3 * i]; my += pos[3 * i + 1]; mz += pos[3 * i + 2];
      }
      out[3 * n] = mx / cnt; out[3 * n + 1] = my / cnt; out[3 * n + 2] = mz / cnt;
    }
  }
}

// upward/real_tree_expansions.py:89-213 (leaf P2M) and :216-364 (M2M by level).
template <typename T>
static void upward(int p, const T* pos, const T* mass, int num_nodes, int num_internal,
                   const int* ranges, const int* left, const int* right, const int* level_off,
                   int num_levels, const T* centers, T* mult) {
  const int C = sh_size(p);
  std::memset(mult, 0, sizeof(T) * (size_t)num_nodes * C);
#pragma omp parallel for schedule(dynamic, 16)
  for (int n = num_internal; n < num_nodes; ++n) {
    T acc[256] = {0}, tmp[256];
    for (int i = ranges[2 * n]; i <= ranges[2 * n + 1]; ++i) {
      T d[3] = {pos[3 * i] - centers[3 * n], pos[3 * i + 1] - centers[3 * n + 1], pos[3 * i + 2] - centers[3 * n + 2]};
      p2m_one(d, mass[i], tmp, p);
      for (int k = 0; k < C; ++k) acc[k] += tmp[k];
    }
    for (int k = 0; k < C; ++k) mult[(size_t)n * C + k] = acc[k];
  }
  for (int lev = num_levels - 1; lev >= 0; --lev) {
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = level_off[lev]; i < level_off[lev + 1]; ++i) {
      T acc[256] = {0}, tmp[256];
      const int ch[2] = {left[i], right[i]};
      for (int c = 0; c < 2; ++c) {
        const int k = ch[c];
        if (k < 0) continue;
        T d[3] = {centers[3 * k] - centers[3 * i], centers[3 * k + 1] - centers[3 * i + 1], centers[3 * k + 2] - centers[3 * i + 2]};
        m2m(mult + (size_t)k * C, d, tmp, p);
        for (int q = 0; q < C; ++q) acc[q] += tmp[q];
      }
      for (int q = 0; q < C; ++q) mult[(size_t)i * C + q] = acc[q];
    }
  }
}

// runtime/kernels/_m2l.py:1483-1793: per pair gather, delta = c[tgt] - c[src],
// segment-sum onto tgt.  Pairs given as CSR over targets.
template <typename T>
static void m2l_accumulate(int p, int num_nodes, const T* mult, const T* centers,
                           const int64_t* far_off, const int* far_src, T* loc) {
  const int C = sh_size(p);
#pragma omp parallel for schedule(dynamic, 8)
  for (int t = 0; t < num_nodes; ++t) {
    T acc[256] = {0}, tmp[256];
    for (int64_t e = far_off[t]; e < far_off[t + 1]; ++e) {
      const int s = far_src[e];
      T d[3] = {centers[3 * t] - centers[3 * s], centers[3 * t + 1] - centers[3 * s + 1], centers[3 * t + 2] - centers[3 * s + 2]};
      m2l(mult + (size_t)s * C, d, tmp, p);
      for (int q = 0; q < C; ++q) acc[q] += tmp[q];
    }
    for (int q = 0; q < C; ++q) loc[(size_t)t * C + q] += acc[q];
  }
}

// runtime/kernels/_l2l.py:210-404: root->leaf cascade, delta = parent - child.
template <typename T>
static void l2l_cascade(int p, const int* left, const int* right, const int* level_off,
                        int num_levels, const T* centers, T* loc) {
  const int C = sh_size(p);
  for (int lev = 0; lev < num_levels; ++lev) {
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = level_off[lev]; i < level_off[lev + 1]; ++i) {
      T tmp[256];
      const int ch[2] = {left[i], right[i]};
      for (int c = 0; c < 2; ++c) {
        const int k = ch[c];
        if (k < 0) continue;
        T d[3] = {centers[3 * i] - centers[3 * k], centers[3 * i + 1] - centers[3 * k + 1], centers[3 * i + 2] - centers[3 * k + 2]};
        l2l(loc + (size_t)i * C, d, tmp, p);
        for (int q = 0; q < C; ++q) loc[(size_t)k * C + q] += tmp[q];
      }
    }
  }
}

// nearfield/_kernels.py:40-141 (self block, diagonal masked) and :251-338
// (pair block): a_i = -G sum m_j (x_i - x_j) rsqrt(r^2+eps^2)^3.
template <typename T>
static void p2p_leaf_pair(const T* pos, const T* mass, int t0, int t1, int s0, int s1, bool self,
                          T G, T eps2, T* acc, T* pot) {
  for (int i = t0; i <= t1; ++i) {
    T ax = 0, ay = 0, az = 0, ph = 0;
    for (int j = s0; j <= s1; ++j) {
      if (self && i == j) continue;
      const T dx = pos[3 * i] - pos[3 * j], dy = pos[3 * i + 1] - pos[3 * j + 1], dz = pos[3 * i + 2] - pos[3 * j + 2];
      const T d2 = dx * dx + dy * dy + dz * dz + eps2;
      const T ir = (T)1 / std::sqrt(d2);
      const T ir3 = ir * ir * ir;
      ax += ir3 * mass[j] * dx; ay += ir3 * mass[j] * dy; az += ir3 * mass[j] * dz;
      ph += ir * mass[j];
    }
    acc[3 * (i - t0)] += -G * ax; acc[3 * (i - t0) + 1] += -G * ay; acc[3 * (i - t0) + 2] += -G * az;
    if (pot) pot[i - t0] += -G * ph;
  }
}

// runtime/kernels/_evaluate.py:769-1172 (near + far assembly, accel = near - G grad)
// and :2106-2484 (L2P per leaf slot, delta = centre - x).
template <typename T>
static void evaluate(int p, const T* pos, const T* mass, int num_nodes, int num_internal,
                     const int* ranges, const T* centers, const T* loc, const int64_t* near_off,
                     const int* near_leaf, T G, T eps2, T* acc_out, T* pot_out, int leaf_lo = 0, int leaf_hi = -1) {
  const int C = sh_size(p);
  const int L = num_nodes - num_internal;
  if (leaf_hi < 0) leaf_hi = L;
#pragma omp parallel for schedule(dynamic, 8)
  for (int lf = leaf_lo; lf < leaf_hi; ++lf) {
    const int node = num_internal + lf;
    const int t0 = ranges[2 * node], t1 = ranges[2 * node + 1];
    const int nt = t1 - t0 + 1;
    std::vector<T> acc(3 * nt, (T)0), pot(nt, (T)0);
    p2p_leaf_pair(pos, mass, t0, t1, t0, t1, true, G, eps2, acc.data(), pot.data());
    for (int64_t e = near_off[lf]; e < near_off[lf + 1]; ++e) {
      const int sn = num_internal + near_leaf[e];
      p2p_leaf_pair(pos, mass, t0, t1, ranges[2 * sn], ranges[2 * sn + 1], false, G, eps2, acc.data(), pot.data());
    }
    for (int i = t0; i <= t1; ++i) {
      T d[3] = {centers[3 * node] - pos[3 * i], centers[3 * node + 1] - pos[3 * i + 1], centers[3 * node + 2] - pos[3 * i + 2]};
      T ph, g[3];
      l2p_one(loc + (size_t)node * C, d, p, &ph, g);
      for (int k = 0; k < 3; ++k) acc_out[3 * i + k] = acc[3 * (i - t0) + k] - G * g[k];
      if (pot_out) pot_out[i] = pot[i - t0] - G * ph;
    }
  }
}

// runtime/kernels/_evaluate.py:1941-2095: target subset.  Each target (sorted
// index) sees its own leaf (minus itself) plus the leaf's neighbour list, and
// the leaf's local expansion.  Output in target order.
template <typename T>
static void evaluate_targets(int p, const T* pos, const T* mass, int num_internal, const int* ranges,
                             const T* centers, const T* loc, const int64_t* near_off, const int* near_leaf,
                             const int* leaf_of, int64_t nt, const int* tsorted, T G, T eps2, T* acc_out, T* pot_out) {
  const int C = sh_size(p);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t q = 0; q < nt; ++q) {
    const int i = tsorted[q];
    const int lf = leaf_of[i];
    const int node = num_internal + lf;
    T acc[3] = {0, 0, 0}, pot = 0;
    // self leaf, excluding i
    p2p_leaf_pair(pos, mass, i, i, ranges[2 * node], ranges[2 * node + 1], true, G, eps2, acc, &pot);
    for (int64_t e = near_off[lf]; e < near_off[lf + 1]; ++e) {
      const int sn = num_internal + near_leaf[e];
      p2p_leaf_pair(pos, mass, i, i, ranges[2 * sn], ranges[2 * sn + 1], false, G, eps2, acc, &pot);
    }
    T d[3] = {centers[3 * node] - pos[3 * i], centers[3 * node + 1] - pos[3 * i + 1], centers[3 * node + 2] - pos[3 * i + 2]};
    T ph, g[3];
    l2p_one(loc + (size_t)node * C, d, p, &ph, g);
    for (int k = 0; k < 3; ++k) acc_out[3 * q + k] = acc[k] - G * g[k];
    if (pot_out) pot_out[q] = pot - G * ph;
  }
}

}  // namespace orc

// ---------------------------------------------------------------------------
// C ABI for the Python test harness (ctypes).
// ---------------------------------------------------------------------------
#define ORC_EXPORT extern "C" __attribute__((visibility("default")))

#define ORC_OPS(T, SFX)                                                                          \
  ORC_EXPORT void oracle_p2m_##SFX(int p, int64_t n, const T* d, const T* m, T* out) {            \
    orc::ensure_tables(p); const int C = orc::sh_size(p);                                        \
    for (int64_t i = 0; i < n; ++i) orc::p2m_one(d + 3 * i, m[i], out + i * C, p);              \
  }                                                                                              \
  ORC_EXPORT void oracle_l2p_##SFX(int p, int64_t n, const T* F, const T* d, T* pot, T* grad) {   \
    orc::ensure_tables(p); const int C = orc::sh_size(p);                                                               \
    for (int64_t i = 0; i < n; ++i) orc::l2p_one(F + i * C, d + 3 * i, p, pot + i, grad + 3 * i); \
  }                                                                                              \
  ORC_EXPORT void oracle_m2m_##SFX(int p, int64_t n, const T* M, const T* d, T* out) {            \
    orc::ensure_tables(p); const int C = orc::sh_size(p);                                                               \
    for (int64_t i = 0; i < n; ++i) orc::m2m(M + i * C, d + 3 * i, out + i * C, p);             \
  }                                                                                              \
  ORC_EXPORT void oracle_l2l_##SFX(int p, int64_t n, const T* M, const T* d, T* out) {            \
    orc::ensure_tables(p); const int C = orc::sh_size(p);                                                               \
    for (int64_t i = 0; i < n; ++i) orc::l2l(M + i * C, d + 3 * i, out + i * C, p);             \
  }                                                                                              \
  ORC_EXPORT void oracle_m2l_##SFX(int p, int64_t n, const T* M, const T* d, T* out) {            \
    orc::ensure_tables(p); const int C = orc::sh_size(p);                                                               \
    for (int64_t i = 0; i < n; ++i) orc::m2l(M + i * C, d + 3 * i, out + i * C, p);             \
  }                                                                                              \
  ORC_EXPORT void oracle_com_##SFX(int64_t N, const T* pos, const T* mass, int num_nodes,         \
                                   const int* ranges, T* out) {                                  \
    orc::com(N, pos, mass, num_nodes, ranges, out);                                              \
  }                                                                                              \
  ORC_EXPORT void oracle_upward_##SFX(int p, const T* pos, const T* mass, int num_nodes,          \
                                      int num_internal, const int* ranges, const int* left,      \
                                      const int* right, const int* level_off, int num_levels,    \
                                      const T* centers, T* mult) {                               \
    orc::ensure_tables(p); orc::upward(p, pos, mass, num_nodes, num_internal, ranges, left, right, level_off,           \
                num_levels, centers, mult);                                                      \
  }                                                                                              \
  ORC_EXPORT void oracle_m2l_accumulate_##SFX(int p, int num_nodes, const T* mult,                \
                                              const T* centers, const int64_t* far_off,          \
                                              const int* far_src, T* loc) {                      \
    orc::ensure_tables(p); orc::m2l_accumulate(p, num_nodes, mult, centers, far_off, far_src, loc);                     \
  }                                                                                              \
  ORC_EXPORT void oracle_l2l_cascade_##SFX(int p, const int* left, const int* right,              \
                                           const int* level_off, int num_levels,                 \
                                           const T* centers, T* loc) {                           \
    orc::ensure_tables(p); orc::l2l_cascade(p, left, right, level_off, num_levels, centers, loc);                       \
  }                                                                                              \
  ORC_EXPORT void oracle_evaluate_##SFX(int p, const T* pos, const T* mass, int num_nodes,        \
                                        int num_internal, const int* ranges, const T* centers,   \
                                        const T* loc, const int64_t* near_off,                   \
                                        const int* near_leaf, T G, T eps2, T* acc, T* pot) {     \
    orc::ensure_tables(p); orc::evaluate(p, pos, mass, num_nodes, num_internal, ranges, centers, loc, near_off,         \
                  near_leaf, G, eps2, acc, pot);                                                 \
  }                                                                                              \
  ORC_EXPORT void oracle_evaluate_range_##SFX(int p, const T* pos, const T* mass, int num_nodes,  \
                                              int num_internal, const int* ranges,               \
                                              const T* centers, const T* loc,                    \
                                              const int64_t* near_off, const int* near_leaf, T G, \
                                              T eps2, int leaf_lo, int leaf_hi, T* acc, T* pot) { \
    orc::ensure_tables(p); orc::evaluate(p, pos, mass, num_nodes, num_internal, ranges, centers, loc, near_off,         \
                  near_leaf, G, eps2, acc, pot, leaf_lo, leaf_hi);                               \
  }                                                                                              \
  ORC_EXPORT void oracle_evaluate_targets_##SFX(                                                 \
      int p, const T* pos, const T* mass, int num_internal, const int* ranges,                   \
      const T* centers, const T* loc, const int64_t* near_off, const int* near_leaf,             \
      const int* leaf_of, int64_t nt, const int* tsorted, T G, T eps2, T* acc, T* pot) {         \
    orc::ensure_tables(p); orc::evaluate_targets(p, pos, mass, num_internal, ranges, centers, loc, near_off, near_leaf, \
                          leaf_of, nt, tsorted, G, eps2, acc, pot);                              \
  }

ORC_OPS(double, f64)
ORC_OPS(float, f32)

// B_U for degree ell (row-major (2l+1)^2), float64.
ORC_EXPORT void oracle_bu(int ell, double* out) {
  std::vector<double> b = orc::real_BU(ell);
  std::memcpy(out, b.data(), sizeof(double) * b.size());
}

// FP64 direct sum over all sources for the given targets (original indices):
// runtime/reference.py:292-330 and bench/validation/mac_error_distribution.py:140-186.
ORC_EXPORT void oracle_direct_f64(int64_t N, const double* pos, const double* mass, int64_t nt,
                                  const int64_t* targets, double G, double eps2, double* acc,
                                  double* pot) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t q = 0; q < nt; ++q) {
    const int64_t i = targets[q];
    double ax = 0, ay = 0, az = 0, ph = 0;
    const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
    for (int64_t j = 0; j < N; ++j) {
      if (j == i) continue;
      const double dx = xi - pos[3 * j], dy = yi - pos[3 * j + 1], dz = zi - pos[3 * j + 2];
      const double d2 = dx * dx + dy * dy + dz * dz + eps2;
      const double ir = 1.0 / std::sqrt(d2);
      const double w = mass[j] * ir * ir * ir;
      ax += w * dx; ay += w * dy; az += w * dz;
      ph += mass[j] * ir;
    }
    acc[3 * q] = -G * ax; acc[3 * q + 1] = -G * ay; acc[3 * q + 2] = -G * az;
    if (pot) pot[q] = -G * ph;
  }
}

ORC_EXPORT int oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}
