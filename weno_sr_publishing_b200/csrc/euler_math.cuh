// FP64 Euler algebra for the 2D path: primitive/conserved maps, physical flux, Roe average,
// characteristic projections, HLLC and FORCE fluxes.
//
// Reference (code/snapshot/): warp_weno5_helpers.py (wh) lines 245-287 (con_to_pri, pri_to_flux),
// 401-435 (force_flux), 598-748 (Roe average, Jacobian values, con_to_char_x/y, char_to_con_x/y);
// for_paper_results/solvers/weno5_hllc.py (HLLC5) lines 22-113 (hllc_flux).
// The formulas and floors are kept exactly; the evaluation order follows the reference so that the
// FP64 path stays within a few ulp of it.
#pragma once
#include <cuda_runtime.h>

namespace wsr {

struct d4 {
  double v[4];
};

// Gas constants with their reciprocals, formed once on the host so that the kernels multiply
// instead of dividing by constants.
struct Gas {
  double g, gm1, inv_gm1, inv_g;
};

inline Gas make_gas(double g) { return Gas{g, g - 1.0, 1.0 / (g - 1.0), 1.0 / g}; }

// 1/x in FP64: the hardware approximation (rcp.approx.ftz.f64, about 20 bits) refined by two
// Newton-Raphson steps r <- r + r (1 - x r), each doubling the number of correct bits, so the result is
// within about 1 ulp of 1/x for normal x. Five instructions instead of a full IEEE division; used where
// the reference divides and last-bit rounding does not matter.
__device__ __forceinline__ double rcp64(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  double e = fma(-x, r, 1.0);
  r = fma(r, e, r);
  e = fma(-x, r, 1.0);
  return fma(r, e, r);
}

__device__ __forceinline__ d4 con_to_pri(const d4& q, double g) {
  d4 w;
  double rho = q.v[0], u = q.v[1] / rho, v = q.v[2] / rho;
  w.v[0] = rho;
  w.v[1] = u;
  w.v[2] = v;
  w.v[3] = (g - 1.0) * (q.v[3] - 0.5 * rho * (u * u + v * v));
  return w;
}

template <int DIR>
__device__ __forceinline__ d4 pri_to_flux(const d4& w, double g) {
  d4 f;
  double rho = w.v[0], u = w.v[1], v = w.v[2], p = w.v[3];
  double e = 0.5 * rho * (u * u + v * v) + p / (g - 1.0);
  if (DIR == 1) {
    f.v[0] = rho * u;
    f.v[1] = rho * u * u + p;
    f.v[2] = rho * u * v;
    f.v[3] = u * (p + e);
  } else {
    f.v[0] = rho * v;
    f.v[1] = rho * u * v;
    f.v[2] = rho * v * v + p;
    f.v[3] = v * (p + e);
  }
  return f;
}

__device__ __forceinline__ double signed_floor(double d, double tiny) {
  return fabs(d) < tiny ? (d < 0.0 ? -tiny : tiny) : d;
}

// HLLC with Davis speeds; rho and p floored at 1e-16; signed floors on the three denominators
// (HLLC5:22-113). Each side's density is inverted once and reused (the reference divides by it five
// times), which changes results only by rounding.
template <int DIR>
__device__ __forceinline__ d4 hllc_flux(const d4& ul0, const d4& ur0, const Gas& gas) {
  const double tiny = 1.0e-16;
  const double g = gas.g, gm1 = gas.gm1, inv_gm1 = gas.inv_gm1;
  const double il = rcp64(ul0.v[0]), ir = rcp64(ur0.v[0]);
  d4 wl, wr;
  wl.v[0] = ul0.v[0];
  wl.v[1] = ul0.v[1] * il;
  wl.v[2] = ul0.v[2] * il;
  wl.v[3] = gm1 * (ul0.v[3] - 0.5 * wl.v[0] * (wl.v[1] * wl.v[1] + wl.v[2] * wl.v[2]));
  wr.v[0] = ur0.v[0];
  wr.v[1] = ur0.v[1] * ir;
  wr.v[2] = ur0.v[2] * ir;
  wr.v[3] = gm1 * (ur0.v[3] - 0.5 * wr.v[0] * (wr.v[1] * wr.v[1] + wr.v[2] * wr.v[2]));
  const double rho_l = fmax(wl.v[0], tiny), rho_r = fmax(wr.v[0], tiny);
  const double irl = wl.v[0] >= tiny ? il : 1.0 / tiny, irr = wr.v[0] >= tiny ? ir : 1.0 / tiny;
  const double p_l = fmax(wl.v[3], tiny), p_r = fmax(wr.v[3], tiny);
  const double a_l = sqrt(g * p_l * irl), a_r = sqrt(g * p_r * irr);
  const double un_l = DIR == 2 ? wl.v[2] : wl.v[1];
  const double un_r = DIR == 2 ? wr.v[2] : wr.v[1];
  const double s_l = fmin(un_l - a_l, un_r - a_r);
  const double s_r = fmax(un_l + a_l, un_r + a_r);
  auto flux_of = [&](const d4& w) {
    d4 f;
    double rho = w.v[0], u = w.v[1], v = w.v[2], p = w.v[3];
    double e = 0.5 * rho * (u * u + v * v) + p * inv_gm1;
    double un = DIR == 1 ? u : v;
    f.v[0] = rho * un;
    f.v[1] = rho * u * un + (DIR == 1 ? p : 0.0);
    f.v[2] = rho * v * un + (DIR == 2 ? p : 0.0);
    f.v[3] = un * (p + e);
    return f;
  };
  if (0.0 <= s_l) return flux_of(wl);
  if (0.0 >= s_r) return flux_of(wr);
  const double denom = signed_floor(rho_l * (s_l - un_l) - rho_r * (s_r - un_r), tiny);
  const double s_star = (p_r - p_l + rho_l * un_l * (s_l - un_l) - rho_r * un_r * (s_r - un_r)) * rcp64(denom);
  const bool right = s_star < 0.0;
  const d4& u_side = right ? ur0 : ul0;
  const d4& w_side = right ? wr : wl;
  const double s_side = right ? s_r : s_l;
  const double irho = right ? irr : irl;
  const d4 f_side = flux_of(w_side);
  const double rho = fmax(w_side.v[0], tiny), u = w_side.v[1], v = w_side.v[2], p = fmax(w_side.v[3], tiny);
  const double un = DIR == 2 ? v : u;
  const double denom_star = signed_floor(s_side - s_star, tiny);
  const double factor = rho * (s_side - un) * rcp64(denom_star);
  d4 us;
  us.v[0] = factor;
  us.v[1] = DIR == 2 ? factor * u : factor * s_star;
  us.v[2] = DIR == 2 ? factor * s_star : factor * v;
  const double denom_side = signed_floor(s_side - un, tiny);
  us.v[3] = factor * ((u_side.v[3] * irho) + (s_star - un) * (s_star + p * rcp64(rho * denom_side)));
  d4 out;
#pragma unroll
  for (int c = 0; c < 4; ++c) out.v[c] = f_side.v[c] + s_side * (us.v[c] - u_side.v[c]);
  return out;
}

// FORCE = 1/2 (Lax-Friedrichs + Richtmyer) with c = dt/h.
template <int DIR>
__device__ __forceinline__ d4 force_flux(const d4& ul0, const d4& ur0, double c, double g) {
  d4 fl = pri_to_flux<DIR>(con_to_pri(ul0, g), g);
  d4 fr = pri_to_flux<DIR>(con_to_pri(ur0, g), g);
  d4 ri_u;
#pragma unroll
  for (int k = 0; k < 4; ++k) ri_u.v[k] = 0.5 * (ul0.v[k] + ur0.v[k]) - 0.5 * c * (fr.v[k] - fl.v[k]);
  d4 ri = pri_to_flux<DIR>(con_to_pri(ri_u, g), g);
  double dx_dt = 1.0 / c;
  d4 out;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    double lf = 0.5 * (fl.v[k] + fr.v[k]) - 0.5 * dx_dt * (ur0.v[k] - ul0.v[k]);
    out.v[k] = 0.5 * (lf + ri.v[k]);
  }
  return out;
}

// Roe-averaged state of two cells, returned directly as the Jacobian values (u, v, a, h) that the
// projections use (wh:598-642 compose roe_average_state and jacobian_state_values).
struct RoeJ {
  double u, v, a, h;
};

__device__ __forceinline__ RoeJ roe_jacobian(const d4& l, const d4& r, const Gas& gas) {
  const double tiny = 1.0e-15;
  const double g = gas.g, gm1 = gas.gm1;
  const double rho_l = fmax(l.v[0], tiny), il = rcp64(rho_l), u_l = l.v[1] * il, v_l = l.v[2] * il, e_l = l.v[3];
  const double p_l = fmax(gm1 * (e_l - 0.5 * rho_l * (u_l * u_l + v_l * v_l)), tiny);
  const double h_l = (e_l + p_l) * il;
  const double rho_r = fmax(r.v[0], tiny), ir = rcp64(rho_r), u_r = r.v[1] * ir, v_r = r.v[2] * ir, e_r = r.v[3];
  const double p_r = fmax(gm1 * (e_r - 0.5 * rho_r * (u_r * u_r + v_r * v_r)), tiny);
  const double h_r = (e_r + p_r) * ir;
  const double sl = sqrt(rho_l), sr = sqrt(rho_r), inv = rcp64(sl + sr);
  const double u = (sl * u_l + sr * u_r) * inv, v = (sl * v_l + sr * v_r) * inv, h = (sl * h_l + sr * h_r) * inv;
  const double rho = sl * sr, q2 = u * u + v * v;
  // roe_average_state encodes (rho, rho u, rho v, E) and jacobian_state_values decodes it; the decoded
  // velocities equal (u, v) up to rounding, so only E -> p -> a is carried through.
  const double e = (rho * h + 0.5 * gm1 * rho * q2) * gas.inv_g;
  const double rr = fmax(rho, tiny);
  RoeJ J;
  J.u = u;
  J.v = v;
  const double p = fmax(gm1 * (e - 0.5 * rr * q2), tiny);
  J.a = sqrt(g * p * rcp64(rr));
  J.h = 0.5 * q2 + J.a * J.a * gas.inv_gm1;
  return J;
}

// Left eigenvector rows (unscaled) for direction DIR, and the common scale (g-1)/(2 a^2).
struct CharL {
  double l[4][4];
  double scale;
};

template <int DIR>
__device__ __forceinline__ CharL char_left(const RoeJ& J, const Gas& gas) {
  CharL L;
  const double gm1 = gas.gm1, ig = gas.inv_gm1, a = J.a, h = J.h, a2 = a * a;
  L.scale = gm1 * rcp64(2.0 * a2);
  const double n = DIR == 1 ? J.u : J.v;  // normal velocity
  const double t = DIR == 1 ? J.v : J.u;  // tangential velocity
  // Component order of q: (rho, m_x, m_y, E); the normal momentum is q[1] for x, q[2] for y.
  const int in = DIR == 1 ? 1 : 2, it = DIR == 1 ? 2 : 1;
  L.l[0][0] = h + a * (n - a) * ig;
  L.l[0][in] = -(n + a * ig);
  L.l[0][it] = -t;
  L.l[0][3] = 1.0;
  L.l[1][0] = -2.0 * h + 4.0 * a2 * ig;
  L.l[1][in] = 2.0 * n;
  L.l[1][it] = 2.0 * t;
  L.l[1][3] = -2.0;
  L.l[2][0] = -2.0 * t * a2 * ig;
  L.l[2][in] = 0.0;
  L.l[2][it] = 2.0 * a2 * ig;
  L.l[2][3] = 0.0;
  L.l[3][0] = h - a * (n + a) * ig;
  L.l[3][in] = -n + a * ig;
  L.l[3][it] = -t;
  L.l[3][3] = 1.0;
  return L;
}

// c_f = (sum_k L[f][k] q[k]) * scale, summed in the reference's term order.
template <int DIR>
__device__ __forceinline__ double project(const CharL& L, int f, const d4& q) {
  if (f == 2) {
    const int it = DIR == 1 ? 2 : 1;
    return (L.l[2][0] * q.v[0] + L.l[2][it] * q.v[it]) * L.scale;
  }
  return (L.l[f][0] * q.v[0] + L.l[f][1] * q.v[1] + L.l[f][2] * q.v[2] + L.l[f][3] * q.v[3]) * L.scale;
}

template <int DIR>
__device__ __forceinline__ d4 char_to_con(const double c[4], const RoeJ& J) {
  double a = J.a, h = J.h;
  double n = DIR == 1 ? J.u : J.v;
  double t = DIR == 1 ? J.v : J.u;
  double q2 = J.u * J.u + J.v * J.v;
  d4 q;
  q.v[0] = c[0] + c[1] + c[3];
  double mn = (n - a) * c[0] + n * c[1] + (n + a) * c[3];
  double mt = t * c[0] + t * c[1] + c[2] + t * c[3];
  q.v[DIR == 1 ? 1 : 2] = mn;
  q.v[DIR == 1 ? 2 : 1] = mt;
  q.v[3] = (h - n * a) * c[0] + 0.5 * q2 * c[1] + t * c[2] + (h + n * a) * c[3];
  return q;
}

}  // namespace wsr
