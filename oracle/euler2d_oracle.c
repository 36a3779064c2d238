/*
 * CPU oracle for the 2D Euler WENO5 (JS / SR) finite-volume step.
 *
 * TEST INFRASTRUCTURE ONLY. This file is a plain-C restatement of the reference's Warp kernels for
 * the 2D path. It is used by the test suite as the parity checker of the CUDA kernels, and by
 * bench.py as the timed CPU baseline. The product path never calls it.
 *
 * Pinned against the reference itself: tests/golden/make_golden.py executes the reference's own
 * Warp source (through a pure-Python stand-in for warp) on small grids and stores the results; the
 * tests check this oracle against those fixtures.
 *
 * Reference files (paths inside the reference project, code/snapshot/):
 *   warp_weno5_helpers.py                        (wh)      Euler algebra, Roe, projections, JS WENO
 *   teacherfree_lab_weno5_v20_distance_balanced/
 *       weno5_rk3_diff_v20_deploy.py             (DEPLOY)  FP64 closure, stage kernels, update
 *       weno5_hllc_refsym.py                     (REFSYM)  FP64 WENO5-SR adapter
 *   teacherfree_lab_weno5_v20_distance_balanced_mlp_f32_fast/warp_mlp_f32/
 *       weno5_rk3_diff_mlp_f32.py                (F32CORE) FP32 closure
 *   for_paper_results/solvers/weno5_hllc.py      (HLLC5)   HLLC flux and the WENO5-JS adapter
 *   for_paper_results/solvers/weno5_hllc_mixed.py (MIXED)  FP32-closure adapter
 *
 * Layout: padded row-major state u[(ny+6)][(nx+6)][4] doubles, conserved (rho, rho u, rho v, E),
 * ghost width 3 (wh:66-87).
 *
 * Build: oracle/build_oracle.py (gcc -O2 -ffp-contract=off -fopenmp -shared).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define GC 3

enum { OR_METHOD_JS = 0, OR_METHOD_SR64 = 1, OR_METHOD_SR32 = 2, OR_METHOD_SRBF16 = 3, OR_METHOD_Z = 4 };
enum { OR_BC_TRANSMISSIVE = 0, OR_BC_PERIODIC = 1, OR_BC_DOUBLE_MACH = 2 };
/* flag OR-ed into the boundary of a stage: the y ghost rows of u_stage are kept as given (a slab of a
 * y-decomposed grid whose halo has been exchanged); x ghosts follow the base boundary */
#define OR_BC_Y_HALO 16
enum { OR_FLUX_HLLC = 0, OR_FLUX_FORCE = 1 };

typedef struct { double v[4]; } vec4;

/* ------------------------------------------------------------------------------------------ */
/* Euler algebra (wh:245-287)                                                                  */
/* ------------------------------------------------------------------------------------------ */

static vec4 con_to_pri(vec4 q, double g) { /* wh:245-251 */
    vec4 w;
    double rho = q.v[0], u = q.v[1] / rho, v = q.v[2] / rho;
    w.v[0] = rho; w.v[1] = u; w.v[2] = v;
    w.v[3] = (g - 1.0) * (q.v[3] - 0.5 * rho * (u * u + v * v));
    return w;
}

static vec4 pri_to_flux(vec4 w, int dir, double g) { /* wh:265-287 */
    vec4 f;
    double rho = w.v[0], u = w.v[1], v = w.v[2], p = w.v[3];
    double e = 0.5 * rho * (u * u + v * v) + p / (g - 1.0);
    if (dir == 1) {
        f.v[0] = rho * u; f.v[1] = rho * u * u + p; f.v[2] = rho * u * v; f.v[3] = u * (p + e);
    } else {
        f.v[0] = rho * v; f.v[1] = rho * u * v; f.v[2] = rho * v * v + p; f.v[3] = v * (p + e);
    }
    return f;
}

/* HLLC flux with Davis wave speeds and 1e-16 floors (HLLC5:22-113). */
static double signed_floor(double d, double tiny) {
    if (fabs(d) < tiny) return d < 0.0 ? -tiny : tiny;
    return d;
}

vec4 or_hllc_flux(vec4 ul0, vec4 ur0, int dir, double g) {
    const double tiny = 1.0e-16;
    vec4 wl = con_to_pri(ul0, g), wr = con_to_pri(ur0, g);
    double rho_l = fmax(wl.v[0], tiny), rho_r = fmax(wr.v[0], tiny);
    double p_l = fmax(wl.v[3], tiny), p_r = fmax(wr.v[3], tiny);
    double a_l = sqrt(g * p_l / rho_l), a_r = sqrt(g * p_r / rho_r);
    double un_l = dir == 2 ? wl.v[2] : wl.v[1];
    double un_r = dir == 2 ? wr.v[2] : wr.v[1];
    double s_l = fmin(un_l - a_l, un_r - a_r);
    double s_r = fmax(un_l + a_l, un_r + a_r);
    vec4 f_l = pri_to_flux(wl, dir, g), f_r = pri_to_flux(wr, dir, g);
    if (0.0 <= s_l) return f_l;
    if (0.0 >= s_r) return f_r;
    double denom = signed_floor(rho_l * (s_l - un_l) - rho_r * (s_r - un_r), tiny);
    double s_star = (p_r - p_l + rho_l * un_l * (s_l - un_l) - rho_r * un_r * (s_r - un_r)) / denom;
    vec4 u_side = ul0, w_side = wl, f_side = f_l;
    double s_side = s_l;
    if (s_star < 0.0) { u_side = ur0; w_side = wr; f_side = f_r; s_side = s_r; }
    double rho = fmax(w_side.v[0], tiny), u = w_side.v[1], v = w_side.v[2], p = fmax(w_side.v[3], tiny);
    double un = dir == 2 ? v : u;
    double denom_star = signed_floor(s_side - s_star, tiny);
    double factor = rho * (s_side - un) / denom_star;
    vec4 us;
    us.v[0] = factor;
    us.v[1] = dir == 2 ? factor * u : factor * s_star;
    us.v[2] = dir == 2 ? factor * s_star : factor * v;
    double denom_side = signed_floor(s_side - un, tiny);
    us.v[3] = factor * ((u_side.v[3] / rho) + (s_star - un) * (s_star + p / (rho * denom_side)));
    vec4 out;
    for (int c = 0; c < 4; ++c) out.v[c] = f_side.v[c] + s_side * (us.v[c] - u_side.v[c]);
    return out;
}

/* FORCE flux = 1/2 (Lax-Friedrichs + Richtmyer), c = dt/h (wh:401-435). */
vec4 or_force_flux(vec4 ul0, vec4 ur0, int dir, double c, double g) {
    vec4 fl = pri_to_flux(con_to_pri(ul0, g), dir, g);
    vec4 fr = pri_to_flux(con_to_pri(ur0, g), dir, g);
    vec4 ri_u, lf, out;
    for (int k = 0; k < 4; ++k) ri_u.v[k] = 0.5 * (ul0.v[k] + ur0.v[k]) - 0.5 * c * (fr.v[k] - fl.v[k]);
    vec4 ri = pri_to_flux(con_to_pri(ri_u, g), dir, g);
    double dx_dt = 1.0 / c;
    for (int k = 0; k < 4; ++k) lf.v[k] = 0.5 * (fl.v[k] + fr.v[k]) - 0.5 * dx_dt * (ur0.v[k] - ul0.v[k]);
    for (int k = 0; k < 4; ++k) out.v[k] = 0.5 * (lf.v[k] + ri.v[k]);
    return out;
}

/* ------------------------------------------------------------------------------------------ */
/* Roe average and characteristic projections (wh:598-748)                                     */
/* ------------------------------------------------------------------------------------------ */

static vec4 roe_average_state(vec4 l, vec4 r, double g) { /* wh:598-628 */
    const double tiny = 1.0e-15;
    double gm1 = g - 1.0;
    double rho_l = fmax(l.v[0], tiny), u_l = l.v[1] / rho_l, v_l = l.v[2] / rho_l, e_l = l.v[3];
    double p_l = fmax(gm1 * (e_l - 0.5 * rho_l * (u_l * u_l + v_l * v_l)), tiny);
    double h_l = (e_l + p_l) / rho_l;
    double rho_r = fmax(r.v[0], tiny), u_r = r.v[1] / rho_r, v_r = r.v[2] / rho_r, e_r = r.v[3];
    double p_r = fmax(gm1 * (e_r - 0.5 * rho_r * (u_r * u_r + v_r * v_r)), tiny);
    double h_r = (e_r + p_r) / rho_r;
    double sl = sqrt(rho_l), sr = sqrt(rho_r), inv = 1.0 / (sl + sr);
    double u = (sl * u_l + sr * u_r) * inv, v = (sl * v_l + sr * v_r) * inv, h = (sl * h_l + sr * h_r) * inv;
    double rho = sl * sr, q2 = u * u + v * v;
    vec4 out;
    out.v[0] = rho; out.v[1] = rho * u; out.v[2] = rho * v;
    out.v[3] = (rho * h + 0.5 * gm1 * rho * q2) / g;
    return out;
}

static vec4 jacobian_state_values(vec4 roe, double g) { /* wh:631-642 -> (u, v, a, h) */
    const double tiny = 1.0e-15;
    double rho = fmax(roe.v[0], tiny), u = roe.v[1] / rho, v = roe.v[2] / rho;
    double gm1 = g - 1.0, q2 = u * u + v * v;
    double p = fmax(gm1 * (roe.v[3] - 0.5 * rho * q2), tiny);
    double a = sqrt(g * p / rho);
    vec4 out;
    out.v[0] = u; out.v[1] = v; out.v[2] = a; out.v[3] = 0.5 * q2 + a * a / gm1;
    return out;
}

/* x: normal = u, tangent = v; y: normal = v, tangent = u (wh:645-748). */
static vec4 con_to_char(vec4 q, vec4 roe, int dir, double g) {
    vec4 jv = jacobian_state_values(roe, g);
    double a = jv.v[2], h = jv.v[3], gm1 = g - 1.0, a2 = a * a, scale = gm1 / (2.0 * a2);
    vec4 c;
    if (dir == 1) {
        double u = jv.v[0], v = jv.v[1];
        c.v[0] = ((h + a * (u - a) / gm1) * q.v[0] - (u + a / gm1) * q.v[1] - v * q.v[2] + q.v[3]) * scale;
        c.v[1] = ((-2.0 * h + 4.0 * a2 / gm1) * q.v[0] + 2.0 * u * q.v[1] + 2.0 * v * q.v[2] - 2.0 * q.v[3]) * scale;
        c.v[2] = (-2.0 * v * a2 / gm1 * q.v[0] + 2.0 * a2 / gm1 * q.v[2]) * scale;
        c.v[3] = ((h - a * (u + a) / gm1) * q.v[0] + (-u + a / gm1) * q.v[1] - v * q.v[2] + q.v[3]) * scale;
    } else {
        double t = jv.v[0], n = jv.v[1];
        c.v[0] = ((h + a * (n - a) / gm1) * q.v[0] - t * q.v[1] - (n + a / gm1) * q.v[2] + q.v[3]) * scale;
        c.v[1] = ((-2.0 * h + 4.0 * a2 / gm1) * q.v[0] + 2.0 * t * q.v[1] + 2.0 * n * q.v[2] - 2.0 * q.v[3]) * scale;
        c.v[2] = (-2.0 * t * a2 / gm1 * q.v[0] + 2.0 * a2 / gm1 * q.v[1]) * scale;
        c.v[3] = ((h - a * (n + a) / gm1) * q.v[0] - t * q.v[1] + (-n + a / gm1) * q.v[2] + q.v[3]) * scale;
    }
    return c;
}

static vec4 char_to_con(vec4 c, vec4 roe, int dir, double g) {
    vec4 jv = jacobian_state_values(roe, g);
    double a = jv.v[2], h = jv.v[3];
    vec4 q;
    if (dir == 1) {
        double u = jv.v[0], v = jv.v[1], q2 = u * u + v * v;
        q.v[0] = c.v[0] + c.v[1] + c.v[3];
        q.v[1] = (u - a) * c.v[0] + u * c.v[1] + (u + a) * c.v[3];
        q.v[2] = v * c.v[0] + v * c.v[1] + c.v[2] + v * c.v[3];
        q.v[3] = (h - u * a) * c.v[0] + 0.5 * q2 * c.v[1] + v * c.v[2] + (h + u * a) * c.v[3];
    } else {
        double t = jv.v[0], n = jv.v[1], q2 = t * t + n * n;
        q.v[0] = c.v[0] + c.v[1] + c.v[3];
        q.v[1] = t * c.v[0] + t * c.v[1] + c.v[2] + t * c.v[3];
        q.v[2] = (n - a) * c.v[0] + n * c.v[1] + (n + a) * c.v[3];
        q.v[3] = (h - n * a) * c.v[0] + 0.5 * q2 * c.v[1] + t * c.v[2] + (h + n * a) * c.v[3];
    }
    return q;
}

/* ------------------------------------------------------------------------------------------ */
/* Candidate stencils (wh:438-446 faces, wh:798-810 Gauss points with the truncated literals)   */
/* ------------------------------------------------------------------------------------------ */

static double stencil_face(double u1, double u2, double u3, int loc) {
    if (loc == 1) return (1.0 / 3.0) * u1 - (7.0 / 6.0) * u2 + (11.0 / 6.0) * u3;
    if (loc == 2) return (-1.0 / 6.0) * u1 + (5.0 / 6.0) * u2 + (1.0 / 3.0) * u3;
    if (loc == 3) return (1.0 / 3.0) * u1 + (5.0 / 6.0) * u2 - (1.0 / 6.0) * u3;
    return (11.0 / 6.0) * u1 - (7.0 / 6.0) * u2 + (1.0 / 3.0) * u3;
}

static double stencil_gauss(double u1, double u2, double u3, int loc) {
    if (loc == 1) return -0.144337567297407 * u1 + 0.577350269189626 * u2 + 0.566987298107780 * u3;
    if (loc == 2) return 0.144337567297406 * u1 + u2 - 0.144337567297407 * u3;
    if (loc == 3) return 1.433012701892220 * u1 - 0.577350269189626 * u2 + 0.144337567297406 * u3;
    if (loc == 4) return 0.144337567297406 * u1 - 0.577350269189626 * u2 + 1.433012701892220 * u3;
    if (loc == 5) return -0.144337567297407 * u1 + u2 + 0.144337567297406 * u3;
    return 0.566987298107781 * u1 + 0.577350269189625 * u2 - 0.144337567297406 * u3;
}

/* Linear weights per head: 0 face lr1, 1 face lr2, 2 Gauss loca1, 3 Gauss loca2 (DEPLOY:134-151). */
static void optimal_weights(int head, double d[3]) {
    double r3 = sqrt(3.0);
    if (head == 0) { d[0] = 0.1; d[1] = 0.6; d[2] = 0.3; }
    else if (head == 1) { d[0] = 0.3; d[1] = 0.6; d[2] = 0.1; }
    else if (head == 2) { d[0] = (210.0 + r3) / 1080.0; d[1] = 11.0 / 18.0; d[2] = (210.0 - r3) / 1080.0; }
    else { d[0] = (210.0 - r3) / 1080.0; d[1] = 11.0 / 18.0; d[2] = (210.0 + r3) / 1080.0; }
}

static void head_candidates(const double q[5], int head, double s[3]) {
    if (head == 0) {
        s[0] = stencil_face(q[0], q[1], q[2], 1); s[1] = stencil_face(q[1], q[2], q[3], 2); s[2] = stencil_face(q[2], q[3], q[4], 3);
    } else if (head == 1) {
        s[0] = stencil_face(q[0], q[1], q[2], 2); s[1] = stencil_face(q[1], q[2], q[3], 3); s[2] = stencil_face(q[2], q[3], q[4], 4);
    } else if (head == 2) {
        s[0] = stencil_gauss(q[0], q[1], q[2], 1); s[1] = stencil_gauss(q[1], q[2], q[3], 2); s[2] = stencil_gauss(q[2], q[3], q[4], 3);
    } else {
        s[0] = stencil_gauss(q[0], q[1], q[2], 4); s[1] = stencil_gauss(q[1], q[2], q[3], 5); s[2] = stencil_gauss(q[2], q[3], q[4], 6);
    }
}

/* Jiang-Shu weights, eps 1e-6, p = 2 (wh:512-570, 813-873). */
static void js_weights(const double q[5], int head, double w[3]) {
    double d[3];
    optimal_weights(head, d);
    double t2 = q[2] - 2.0 * q[3] + q[4], u2 = 3.0 * q[2] - 4.0 * q[3] + q[4];
    double t1 = q[1] - 2.0 * q[2] + q[3], u1 = q[1] - q[3];
    double t0 = q[0] - 2.0 * q[1] + q[2], u0 = q[0] - 4.0 * q[1] + 3.0 * q[2];
    double b2 = (13.0 / 12.0) * t2 * t2 + 0.25 * u2 * u2;
    double b1 = (13.0 / 12.0) * t1 * t1 + 0.25 * u1 * u1;
    double b0 = (13.0 / 12.0) * t0 * t0 + 0.25 * u0 * u0;
    double i0 = 1.0 / (1.0e-6 + b0), i1 = 1.0 / (1.0e-6 + b1), i2 = 1.0 / (1.0e-6 + b2);
    double a0 = d[0] * i0 * i0, a1 = d[1] * i1 * i1, a2 = d[2] * i2 * i2;
    double s = a0 + a1 + a2;
    w[0] = a0 / s; w[1] = a1 / s; w[2] = a2 / s;
}

/* WENO-Z, Borges et al. p = 2, eps = h^2 of the reconstruction direction
 * (weno_z_borges_p2_results/weno5_helpers_z.py:545-574, 853-879). */
static void z_weights(const double q[5], int head, double eps, double w[3]) {
    double d[3];
    optimal_weights(head, d);
    double t2 = q[2] - 2.0 * q[3] + q[4], u2 = 3.0 * q[2] - 4.0 * q[3] + q[4];
    double t1 = q[1] - 2.0 * q[2] + q[3], u1 = q[1] - q[3];
    double t0 = q[0] - 2.0 * q[1] + q[2], u0 = q[0] - 4.0 * q[1] + 3.0 * q[2];
    double b2 = (13.0 / 12.0) * t2 * t2 + 0.25 * u2 * u2;
    double b1 = (13.0 / 12.0) * t1 * t1 + 0.25 * u1 * u1;
    double b0 = (13.0 / 12.0) * t0 * t0 + 0.25 * u0 * u0;
    double tau = fabs(b0 - b2);
    double r0 = tau / (b0 + eps), r1 = tau / (b1 + eps), r2 = tau / (b2 + eps);
    double a0 = d[0] * (1.0 + r0 * r0), a1 = d[1] * (1.0 + r1 * r1), a2 = d[2] * (1.0 + r2 * r2);
    double s = a0 + a1 + a2;
    w[0] = a0 / s; w[1] = a1 / s; w[2] = a2 / s;
}

/* ------------------------------------------------------------------------------------------ */
/* Closure: features (DEPLOY:76-120), plateau (DEPLOY:123-131), MLP (DEPLOY:154-205;            */
/* F32CORE:152-203), reflection-averaged weights (DEPLOY:208-279; F32CORE:206-283)             */
/* ------------------------------------------------------------------------------------------ */

/* Packed parameter layout, shared with the CUDA path: w1[5][10] b1[10] w2[10][6] b2[6]
 * w3[6][6] b3[6] w4[6][3] b4[3] (row-major [in][out]) = 189 values. */
#define P_W1 0
#define P_B1 50
#define P_W2 60
#define P_B2 120
#define P_W3 126
#define P_B3 162
#define P_W4 168
#define P_B4 186
#define N_PARAMS5 189

static void raw_sensors(const double q[5], double out[4]) {
    double d20 = q[0] - 2.0 * q[1] + q[2], d21 = q[1] - 2.0 * q[2] + q[3], d22 = q[2] - 2.0 * q[3] + q[4];
    out[0] = (13.0 / 12.0) * fabs(d20) + 0.25 * fabs(q[0] - 4.0 * q[1] + 3.0 * q[2]);
    out[1] = (13.0 / 12.0) * fabs(d21) + 0.25 * fabs(q[1] - q[3]);
    out[2] = (13.0 / 12.0) * fabs(d22) + 0.25 * fabs(3.0 * q[2] - 4.0 * q[3] + q[4]);
    const double eps = 1.0e-15;
    double g0 = fabs(d20) / (fabs(q[1] - q[0]) + fabs(q[2] - q[1]) + eps);
    double g1 = fabs(d21) / (fabs(q[2] - q[1]) + fabs(q[3] - q[2]) + eps);
    double g2 = fabs(d22) / (fabs(q[3] - q[2]) + fabs(q[4] - q[3]) + eps);
    out[3] = fmin(1.0, fmax(fmax(g0, g1), g2));
}

static double q_scale_of(const double q[5]) {
    double s = fmax(fmax(fmax(fabs(q[0]), fabs(q[1])), fmax(fabs(q[2]), fabs(q[3]))), fabs(q[4]));
    return fmax(s, 1.0);
}

/* Effective scale feature is clip((log10(rel) + 4)/4, 0, 1) (DEPLOY:96-120). */
void or_weno5_features(const double q[5], double f[5]) {
    double raw[4];
    raw_sensors(q, raw);
    double dmax = fmax(fmax(raw[0], raw[1]), raw[2]);
    double inv = 1.0 / fmax(dmax, 1.0e-15);
    double rel = fmax(dmax / q_scale_of(q), 1.0e-30);
    double l10 = log(rel) / log(10.0);
    double s = (l10 + 4.0) / 4.0;
    s = fmin(1.0, fmax(0.0, s));
    f[0] = raw[0] * inv; f[1] = raw[1] * inv; f[2] = raw[2] * inv; f[3] = raw[3]; f[4] = s;
}

static int plateau_detected(const double q[5]) {
    double raw[4];
    raw_sensors(q, raw);
    double dmax = fmax(fmax(raw[0], raw[1]), raw[2]);
    return dmax <= 1.0e-13 * q_scale_of(q);
}

void or_mlp_ratios_f64(const double x[5], const double *P, double r[3]) {
    double h1[10], h2[6], h3[6];
    for (int o = 0; o < 10; ++o) {
        double z = P[P_B1 + o];
        for (int k = 0; k < 5; ++k) z = z + x[k] * P[P_W1 + k * 10 + o];
        h1[o] = z / (1.0 + exp(-z));
    }
    for (int o = 0; o < 6; ++o) {
        double z = P[P_B2 + o];
        for (int k = 0; k < 10; ++k) z = z + h1[k] * P[P_W2 + k * 6 + o];
        h2[o] = z / (1.0 + exp(-z));
    }
    for (int o = 0; o < 6; ++o) {
        double z = P[P_B3 + o];
        for (int k = 0; k < 6; ++k) z = z + h2[k] * P[P_W3 + k * 6 + o];
        h3[o] = z / (1.0 + exp(-z));
    }
    double raw[3];
    for (int o = 0; o < 3; ++o) {
        double z = P[P_B4 + o];
        for (int k = 0; k < 6; ++k) z = z + h3[k] * P[P_W4 + k * 3 + o];
        raw[o] = 6.0 * tanh(z / 6.0);
    }
    double m = fmax(fmax(raw[0], raw[1]), raw[2]);
    double e0 = exp(raw[0] - m), e1 = exp(raw[1] - m), e2 = exp(raw[2] - m);
    double inv = 1.0 / (e0 + e1 + e2);
    r[0] = e0 * inv; r[1] = e1 * inv; r[2] = e2 * inv;
}

void or_mlp_ratios_f32(const float x[5], const float *P, float r[3]) {
    float h1[10], h2[6], h3[6];
    for (int o = 0; o < 10; ++o) {
        float z = P[P_B1 + o];
        for (int k = 0; k < 5; ++k) z = z + x[k] * P[P_W1 + k * 10 + o];
        h1[o] = z / (1.0f + expf(-z));
    }
    for (int o = 0; o < 6; ++o) {
        float z = P[P_B2 + o];
        for (int k = 0; k < 10; ++k) z = z + h1[k] * P[P_W2 + k * 6 + o];
        h2[o] = z / (1.0f + expf(-z));
    }
    for (int o = 0; o < 6; ++o) {
        float z = P[P_B3 + o];
        for (int k = 0; k < 6; ++k) z = z + h2[k] * P[P_W3 + k * 6 + o];
        h3[o] = z / (1.0f + expf(-z));
    }
    float raw[3];
    for (int o = 0; o < 3; ++o) {
        float z = P[P_B4 + o];
        for (int k = 0; k < 6; ++k) z = z + h3[k] * P[P_W4 + k * 3 + o];
        raw[o] = 6.0f * tanhf(z / 6.0f);
    }
    float m = fmaxf(fmaxf(raw[0], raw[1]), raw[2]);
    float e0 = expf(raw[0] - m), e1 = expf(raw[1] - m), e2 = expf(raw[2] - m);
    float inv = 1.0f / (e0 + e1 + e2);
    r[0] = e0 * inv; r[1] = e1 * inv; r[2] = e2 * inv;
}

/* BF16 closure (no counterpart in the reference): inputs, parameters and hidden activations are
 * rounded to bfloat16 (round to nearest even) before each layer; products accumulate in FP32;
 * activation functions and the softmax run in FP32. */
static float bf16_round(float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return x; /* inf/nan */
    uint32_t lsb = (u >> 16) & 1u;
    u = (u + 0x7fffu + lsb) & 0xffff0000u;
    float y;
    memcpy(&y, &u, 4);
    return y;
}

void or_mlp_ratios_bf16(const float x_in[5], const float *P, float r[3]) {
    float x[5], h1[10], h2[6], h3[6];
    for (int k = 0; k < 5; ++k) x[k] = bf16_round(x_in[k]);
    for (int o = 0; o < 10; ++o) {
        float z = bf16_round(P[P_B1 + o]);
        for (int k = 0; k < 5; ++k) z = z + x[k] * bf16_round(P[P_W1 + k * 10 + o]);
        h1[o] = bf16_round(z / (1.0f + expf(-z)));
    }
    for (int o = 0; o < 6; ++o) {
        float z = bf16_round(P[P_B2 + o]);
        for (int k = 0; k < 10; ++k) z = z + h1[k] * bf16_round(P[P_W2 + k * 6 + o]);
        h2[o] = bf16_round(z / (1.0f + expf(-z)));
    }
    for (int o = 0; o < 6; ++o) {
        float z = bf16_round(P[P_B3 + o]);
        for (int k = 0; k < 6; ++k) z = z + h2[k] * bf16_round(P[P_W3 + k * 6 + o]);
        h3[o] = bf16_round(z / (1.0f + expf(-z)));
    }
    float raw[3];
    for (int o = 0; o < 3; ++o) {
        float z = bf16_round(P[P_B4 + o]);
        for (int k = 0; k < 6; ++k) z = z + h3[k] * bf16_round(P[P_W4 + k * 3 + o]);
        raw[o] = 6.0f * tanhf(z / 6.0f);
    }
    float m = fmaxf(fmaxf(raw[0], raw[1]), raw[2]);
    float e0 = expf(raw[0] - m), e1 = expf(raw[1] - m), e2 = expf(raw[2] - m);
    float inv = 1.0f / (e0 + e1 + e2);
    r[0] = e0 * inv; r[1] = e1 * inv; r[2] = e2 * inv;
}

/* Closure weights for one stencil and head. P64 is the FP64 parameter block, P32 the FP32 one
 * (used by the FP32 and BF16 closures). */
void or_closure_weights(const double q[5], int head, int method, const double *P64, const float *P32,
                        double w[3]) {
    double d[3];
    optimal_weights(head, d);
    if (method == OR_METHOD_JS) { js_weights(q, head, w); return; }
    if (plateau_detected(q)) { w[0] = d[0]; w[1] = d[1]; w[2] = d[2]; return; }
    double qr[5] = {q[4], q[3], q[2], q[1], q[0]};
    double fd[5], fr[5], rd[3], rr[3];
    or_weno5_features(q, fd);
    or_weno5_features(qr, fr);
    if (method == OR_METHOD_SR64) {
        or_mlp_ratios_f64(fd, P64, rd);
        or_mlp_ratios_f64(fr, P64, rr);
    } else {
        float xd[5], xr[5], od[3], orr[3];
        for (int k = 0; k < 5; ++k) { xd[k] = (float)fd[k]; xr[k] = (float)fr[k]; }
        if (method == OR_METHOD_SR32) { or_mlp_ratios_f32(xd, P32, od); or_mlp_ratios_f32(xr, P32, orr); }
        else { or_mlp_ratios_bf16(xd, P32, od); or_mlp_ratios_bf16(xr, P32, orr); }
        for (int k = 0; k < 3; ++k) { rd[k] = (double)od[k]; rr[k] = (double)orr[k]; }
    }
    double b0 = 0.5 * (rd[0] + rr[2]), b1 = 0.5 * (rd[1] + rr[1]), b2 = 0.5 * (rd[2] + rr[0]);
    double i0 = 1.0 / (3.0 * b0 + 1.0e-12), i1 = 1.0 / (3.0 * b1 + 1.0e-12), i2 = 1.0 / (3.0 * b2 + 1.0e-12);
    double a0 = d[0] * (i0 * i0), a1 = d[1] * (i1 * i1), a2 = d[2] * (i2 * i2);
    double inv = 1.0 / fmax(a0 + a1 + a2, 1.0e-300);
    w[0] = a0 * inv; w[1] = a1 * inv; w[2] = a2 * inv;
}

double or_reconstruct(const double q[5], int head, int method, const double *P64, const float *P32) {
    double w[3], s[3];
    or_closure_weights(q, head, method, P64, P32, w);
    head_candidates(q, head, s);
    return w[0] * s[0] + w[1] * s[1] + w[2] * s[2];
}

/* The reconstruction with the grid spacing h of its direction (used by WENO-Z only). */
double or_reconstruct_h(const double q[5], int head, int method, const double *P64, const float *P32, double h) {
    if (method != OR_METHOD_Z) return or_reconstruct(q, head, method, P64, P32);
    double w[3], s[3];
    z_weights(q, head, h * h, w);
    head_candidates(q, head, s);
    return w[0] * s[0] + w[1] * s[1] + w[2] * s[2];
}

/* ------------------------------------------------------------------------------------------ */
/* Stage (REFSYM:298-435 / MIXED:121-168 / HLLC5:294-358)                                      */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
    int nx, ny, method, bc, flux;
    double dx, dy, gamma;
    const double *P64;
    const float *P32;
    double bt; /* boundary time of the stage (double-Mach only) */
    int y_halo; /* y ghost rows taken as stored (OR_BC_Y_HALO) */
} or_cfg;

static inline vec4 load4(const double *a, int nxt, int j, int i) {
    vec4 q;
    memcpy(q.v, a + ((size_t)j * nxt + i) * 4, sizeof(q.v));
    return q;
}
static inline void store4(double *a, int nxt, int j, int i, vec4 q) {
    memcpy(a + ((size_t)j * nxt + i) * 4, q.v, sizeof(q.v));
}

/* Double-Mach reflection (REFSYM:26-124): a Mach-10 shock through (1/6, 0) at 60 degrees to the wall.
 * The exact pre/post-shock state fills the top ghost rows (at the shock position of time t), the left ghost
 * columns and the bottom ghost rows left of x = 1/6; the bottom ghost rows right of it reflect the interior
 * (v negated); the right ghost columns copy the last interior column. */
static vec4 double_mach_state(double x, double y, double t, double g) {
    double r3 = sqrt(3.0);
    double shock_x = 1.0 / 6.0 + y / r3 + 20.0 * t / r3;
    double rho, u, v, p;
    if (x < shock_x) { rho = 8.0; u = 8.25 * r3 * 0.5; v = -8.25 * 0.5; p = 116.5; }
    else { rho = 1.4; u = 0.0; v = 0.0; p = 1.0; }
    vec4 q = {{rho, rho * u, rho * v, 0.5 * rho * (u * u + v * v) + p / (g - 1.0)}};
    return q;
}

static void apply_double_mach(double *a, const or_cfg *c) {
    int nx = c->nx, ny = c->ny, nxt = nx + 2 * GC, nyt = ny + 2 * GC;
    for (int j = 0; j < nyt; ++j) {
        for (int i = 0; i < nxt; ++i) {
            int in_x = i >= GC && i < nx + GC, in_y = j >= GC && j < ny + GC;
            if (in_x && in_y) continue;
            double x = ((double)(i - GC) + 0.5) * c->dx, y = ((double)(j - GC) + 0.5) * c->dy;
            if (j >= ny + GC) {
                store4(a, nxt, j, i, double_mach_state(x, y, c->bt, c->gamma));
            } else if (j < GC) {
                if (x < 1.0 / 6.0) {
                    store4(a, nxt, j, i, double_mach_state(x, 0.0, c->bt, c->gamma));
                } else {
                    int si = i < GC ? GC : (i >= nx + GC ? nx + GC - 1 : i);
                    vec4 q = load4(a, nxt, 2 * GC - 1 - j, si);
                    q.v[2] = -q.v[2];
                    store4(a, nxt, j, i, q);
                }
            } else if (i < GC) {
                store4(a, nxt, j, i, double_mach_state(x, y, c->bt, c->gamma));
            } else {
                store4(a, nxt, j, i, load4(a, nxt, j, nx + GC - 1));
            }
        }
    }
}

/* copy_transmissive_boundary_kernel / copy_periodic_boundary_kernel (DEPLOY:371-408) */
static void apply_bc(const double *src, double *dst, const or_cfg *c) {
    int nxt = c->nx + 2 * GC, nyt = c->ny + 2 * GC;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < nyt; ++j) {
        for (int i = 0; i < nxt; ++i) {
            int si = i, sj = j;
            if (c->bc != OR_BC_PERIODIC) {
                if (i < GC) si = GC; else if (i >= c->nx + GC) si = c->nx + GC - 1;
                if (j < GC) sj = GC; else if (j >= c->ny + GC) sj = c->ny + GC - 1;
            } else {
                if (i < GC) si = i + c->nx; else if (i >= c->nx + GC) si = i - c->nx;
                if (j < GC) sj = j + c->ny; else if (j >= c->ny + GC) sj = j - c->ny;
            }
            if (c->y_halo) sj = j;
            store4(dst, nxt, j, i, load4(src, nxt, sj, si));
        }
    }
    if (c->bc == OR_BC_DOUBLE_MACH) apply_double_mach(dst, c);
}

/* Characteristic normal reconstruction of the cell centred on stencil q[2]: left face (lr=2,
 * Roe(q1,q2)) and right face (lr=1, Roe(q2,q3)) (DEPLOY:479-592, wh:766-795). */
static void normal_recon(const vec4 q[5], int dir, const or_cfg *c, vec4 *face_l, vec4 *face_r) {
    for (int side = 0; side < 2; ++side) {
        int head = side == 0 ? 1 : 0; /* left face uses lr=2 -> head 1 */
        vec4 roe = side == 0 ? roe_average_state(q[1], q[2], c->gamma) : roe_average_state(q[2], q[3], c->gamma);
        vec4 ch[5];
        for (int k = 0; k < 5; ++k) ch[k] = con_to_char(q[k], roe, dir, c->gamma);
        vec4 cf;
        for (int f = 0; f < 4; ++f) {
            double s[5] = {ch[0].v[f], ch[1].v[f], ch[2].v[f], ch[3].v[f], ch[4].v[f]};
            cf.v[f] = or_reconstruct_h(s, head, c->method, c->P64, c->P32, dir == 1 ? c->dx : c->dy);
        }
        vec4 out = char_to_con(cf, roe, dir, c->gamma);
        if (side == 0) *face_l = out; else *face_r = out;
    }
}

static vec4 riemann(vec4 ul, vec4 ur, int dir, double dt_h, const or_cfg *c) {
    if (c->flux == OR_FLUX_FORCE) return or_force_flux(ul, ur, dir, dt_h, c->gamma);
    return or_hllc_flux(ul, ur, dir, c->gamma);
}

/* Work arrays: bc, xl, xr, yl, yr, fx1, fx2, fy1, fy2 -- each padded-shape. */
typedef struct { double *bc, *xl, *xr, *yl, *yr, *fx1, *fx2, *fy1, *fy2; } or_stage_buf;

static void stage(const double *u_stage, const double *u0, double *u_out, double dt, int rk, const or_cfg *c,
                  or_stage_buf *b) {
    int nx = c->nx, ny = c->ny, nxt = nx + 2 * GC;
    double dt_dx = dt / c->dx, dt_dy = dt / c->dy;
    apply_bc(u_stage, b->bc, c);
    /* x-normal: rows j in [0, ny+6), centre column i+2, i in [0, nx+2) */
#pragma omp parallel for schedule(dynamic, 1)
    for (int j = 0; j < ny + 6; ++j) {
        for (int i = 0; i < nx + 2; ++i) {
            vec4 q[5], fl, fr;
            for (int k = 0; k < 5; ++k) q[k] = load4(b->bc, nxt, j, i + k);
            normal_recon(q, 1, c, &fl, &fr);
            store4(b->xl, nxt, j, i, fl);
            store4(b->xr, nxt, j, i, fr);
        }
    }
    /* y-normal: rows j in [0, ny+2) (centre row j+2), columns i in [0, nx+6) */
#pragma omp parallel for schedule(dynamic, 1)
    for (int j = 0; j < ny + 2; ++j) {
        for (int i = 0; i < nx + 6; ++i) {
            vec4 q[5], fl, fr;
            for (int k = 0; k < 5; ++k) q[k] = load4(b->bc, nxt, j + k, i);
            normal_recon(q, 2, c, &fl, &fr);
            store4(b->yl, nxt, j, i, fl);
            store4(b->yr, nxt, j, i, fr);
        }
    }
    /* x faces (REFSYM:127-195, HLLC5:130-158): face (j, i) between interior cells i-1 and i */
#pragma omp parallel for schedule(dynamic, 1)
    for (int j = 0; j < ny; ++j) {
        for (int i = 0; i < nx + 1; ++i) {
            for (int loca = 1; loca <= 2; ++loca) {
                int head = loca == 1 ? 2 : 3;
                vec4 ul, ur;
                for (int comp = 0; comp < 4; ++comp) {
                    double sr[5], sl[5];
                    for (int k = 0; k < 5; ++k) {
                        sr[k] = b->xl[((size_t)(j + 1 + k) * nxt + (i + 1)) * 4 + comp];
                        sl[k] = b->xr[((size_t)(j + 1 + k) * nxt + i) * 4 + comp];
                    }
                    ur.v[comp] = or_reconstruct_h(sr, head, c->method, c->P64, c->P32, c->dy);
                    ul.v[comp] = or_reconstruct_h(sl, head, c->method, c->P64, c->P32, c->dy);
                }
                vec4 f = riemann(ul, ur, 1, dt_dx, c);
                for (int k = 0; k < 4; ++k) f.v[k] *= dt_dx;
                store4(loca == 1 ? b->fx1 : b->fx2, nxt, j, i, f);
            }
        }
    }
    /* y faces (REFSYM:198-266, HLLC5:161-189): face (j, i) between interior rows j-1 and j */
#pragma omp parallel for schedule(dynamic, 1)
    for (int j = 0; j < ny + 1; ++j) {
        for (int i = 0; i < nx; ++i) {
            for (int loca = 1; loca <= 2; ++loca) {
                int head = loca == 1 ? 2 : 3;
                vec4 ul, ur;
                for (int comp = 0; comp < 4; ++comp) {
                    double sr[5], sl[5];
                    for (int k = 0; k < 5; ++k) {
                        sr[k] = b->yl[((size_t)(j + 1) * nxt + (i + 1 + k)) * 4 + comp];
                        sl[k] = b->yr[((size_t)j * nxt + (i + 1 + k)) * 4 + comp];
                    }
                    ur.v[comp] = or_reconstruct_h(sr, head, c->method, c->P64, c->P32, c->dx);
                    ul.v[comp] = or_reconstruct_h(sl, head, c->method, c->P64, c->P32, c->dx);
                }
                vec4 f = riemann(ul, ur, 2, dt_dy, c);
                for (int k = 0; k < 4; ++k) f.v[k] *= dt_dy;
                store4(loca == 1 ? b->fy1 : b->fy2, nxt, j, i, f);
            }
        }
    }
    /* update_rk3_out_kernel (DEPLOY:1027-1056) */
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; ++j) {
        for (int i = 0; i < nx; ++i) {
            int jj = j + GC, ii = i + GC;
            for (int comp = 0; comp < 4; ++comp) {
#define F(a, jy, ix) (a)[((size_t)(jy) * nxt + (ix)) * 4 + comp]
                double fxr = F(b->fx1, j, i + 1) + F(b->fx2, j, i + 1);
                double fxl = F(b->fx1, j, i) + F(b->fx2, j, i);
                double fyt = F(b->fy1, j + 1, i) + F(b->fy2, j + 1, i);
                double fyb = F(b->fy1, j, i) + F(b->fy2, j, i);
                double rhs = F(b->bc, jj, ii) - 0.5 * (fxr - fxl) - 0.5 * (fyt - fyb);
                double out;
                if (rk == 1) out = rhs;
                else if (rk == 2) out = 0.75 * F(u0, jj, ii) + 0.25 * rhs;
                else out = (1.0 / 3.0) * F(u0, jj, ii) + (2.0 / 3.0) * rhs;
                F(u_out, jj, ii) = out;
#undef F
            }
        }
    }
}

/* compute_max_speed_kernel + host max (wh:876-897, 189-207) */
double or_euler2d_max_speed(const double *u, int nx, int ny, double gamma) {
    int nxt = nx + 2 * GC;
    double m = 0.0;
#pragma omp parallel for reduction(max : m) schedule(static)
    for (int j = 0; j < ny; ++j) {
        for (int i = 0; i < nx; ++i) {
            const double *q = u + ((size_t)(j + GC) * nxt + (i + GC)) * 4;
            double rho = fmax(q[0], 1.0e-15), vx = q[1] / rho, vy = q[2] / rho;
            double p = (gamma - 1.0) * (q[3] - 0.5 * rho * (vx * vx + vy * vy));
            p = fmax(p, 1.0e-15);
            double a = sqrt(gamma * p / rho);
            double s = fmax(fabs(vx) + a, fabs(vy) + a);
            if (s > m) m = s;
        }
    }
    return m;
}

static size_t padded_len(int nx, int ny) { return (size_t)(nx + 2 * GC) * (ny + 2 * GC) * 4; }

static int alloc_stage(or_stage_buf *b, size_t n) {
    double **p[9] = {&b->bc, &b->xl, &b->xr, &b->yl, &b->yr, &b->fx1, &b->fx2, &b->fy1, &b->fy2};
    for (int k = 0; k < 9; ++k) {
        *p[k] = (double *)calloc(n, sizeof(double));
        if (!*p[k]) return -1;
    }
    return 0;
}
static void free_stage(or_stage_buf *b) {
    free(b->bc); free(b->xl); free(b->xr); free(b->yl); free(b->yr);
    free(b->fx1); free(b->fx2); free(b->fy1); free(b->fy2);
}

/* One SSPRK3 stage: u_out(interior) from u_stage and u0, with the boundary evaluated at boundary_time
 * (the double-Mach boundary depends on it). Returns 0 on success. */
int or_euler2d_stage_at(const double *u_stage, const double *u0, double *u_out, int nx, int ny, double dx,
                        double dy, double gamma, double dt, int rk, int method, int bc, int flux,
                        const double *P64, const float *P32, double boundary_time) {
    or_cfg c = {nx, ny, method, bc & ~OR_BC_Y_HALO, flux, dx, dy, gamma, P64, P32, boundary_time,
                (bc & OR_BC_Y_HALO) != 0};
    or_stage_buf b;
    if (alloc_stage(&b, padded_len(nx, ny))) { free_stage(&b); return -1; }
    stage(u_stage, u0, u_out, dt, rk, &c, &b);
    free_stage(&b);
    return 0;
}

int or_euler2d_stage(const double *u_stage, const double *u0, double *u_out, int nx, int ny, double dx,
                     double dy, double gamma, double dt, int rk, int method, int bc, int flux,
                     const double *P64, const float *P32) {
    return or_euler2d_stage_at(u_stage, u0, u_out, nx, ny, dx, dy, gamma, dt, rk, method, bc, flux, P64, P32, 0.0);
}

/* run_to_time (REFSYM:462-544, MIXED:185-212, HLLC5:386-410). State buffers follow the reference:
 * u0 holds the initial padded state; u1..u3 start at zero and only their interiors are written;
 * u0 and u3 swap after each step. On return `out` holds the final padded array the reference
 * returns (its ghost cells depend on the parity of the step count, as in the reference).
 * Writes up to max_steps dt values; returns the step count or -1 on allocation failure.
 * fixed_steps > 0 runs exactly that many full-CFL steps (t_end ignored), for timing. */
int or_euler2d_run(const double *initial, double *out, int nx, int ny, double dx, double dy, double gamma,
                   double cfl, double t_end, int method, int bc, int flux, const double *P64, const float *P32,
                   int check_health, int fixed_steps, double *dts, int max_steps, double *t_out) {
    size_t n = padded_len(nx, ny);
    or_cfg c = {nx, ny, method, bc, flux, dx, dy, gamma, P64, P32};
    double *u[4];
    for (int k = 0; k < 4; ++k) u[k] = (double *)calloc(n, sizeof(double));
    or_stage_buf b;
    int bad = alloc_stage(&b, n);
    for (int k = 0; k < 4; ++k) bad |= u[k] == NULL;
    if (bad) { for (int k = 0; k < 4; ++k) free(u[k]); free_stage(&b); return -1; }
    memcpy(u[0], initial, n * sizeof(double));
    double t = 0.0;
    int step = 0;
    double hmin = dx < dy ? dx : dy;
    while (fixed_steps > 0 ? step < fixed_steps : t < t_end - 1.0e-14) {
        double ms = or_euler2d_max_speed(u[0], nx, ny, gamma);
        double dt = ms < 1.0e-15 ? 1.0e10 : cfl * hmin / ms;
        if (fixed_steps <= 0 && t_end - t < dt) dt = t_end - t;
        if (!isfinite(dt) || dt <= 0.0) break;
        /* boundary times of the three stages: t, t + dt, t + dt/2 (REFSYM:479-527) */
        c.bt = t;
        stage(u[0], u[0], u[1], dt, 1, &c, &b);
        c.bt = t + dt;
        stage(u[1], u[0], u[2], dt, 2, &c, &b);
        c.bt = t + 0.5 * dt;
        stage(u[2], u[0], u[3], dt, 3, &c, &b);
        double *tmp = u[0]; u[0] = u[3]; u[3] = tmp;
        t += dt;
        if (step < max_steps && dts) dts[step] = dt;
        ++step;
        if (check_health && (step == 1 || t >= t_end - 1.0e-14)) {
            int unhealthy = 0;
            for (int j = 0; j < ny && !unhealthy; ++j)
                for (int i = 0; i < nx; ++i) {
                    const double *q = u[0] + ((size_t)(j + GC) * (nx + 2 * GC) + (i + GC)) * 4;
                    double rho = fmax(q[0], 1.0e-15);
                    double p = (gamma - 1.0) * (q[3] - 0.5 * rho * ((q[1] / rho) * (q[1] / rho) + (q[2] / rho) * (q[2] / rho)));
                    /* wh.interior_stats (wh:210-224): NaN count, and p <= 0 with rho floored */
                    if (isnan(q[0]) || isnan(q[1]) || isnan(q[2]) || isnan(q[3]) || p <= 0.0) {
                        unhealthy = 1;
                        break;
                    }
                }
            if (unhealthy) break;
        }
    }
    memcpy(out, u[0], n * sizeof(double));
    if (t_out) *t_out = t;
    for (int k = 0; k < 4; ++k) free(u[k]);
    free_stage(&b);
    return step;
}

int or_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Thin wrappers with flat arrays for ctypes. */
void or_hllc_flux_flat(const double *ul, const double *ur, int dir, double g, double *out) {
    vec4 a, b;
    memcpy(a.v, ul, 32); memcpy(b.v, ur, 32);
    vec4 f = or_hllc_flux(a, b, dir, g);
    memcpy(out, f.v, 32);
}

void or_force_flux_flat(const double *ul, const double *ur, int dir, double c, double g, double *out) {
    vec4 a, b;
    memcpy(a.v, ul, 32); memcpy(b.v, ur, 32);
    vec4 f = or_force_flux(a, b, dir, c, g);
    memcpy(out, f.v, 32);
}

void or_closure_weights_batch(const double *q, int n, int head, int method, const double *P64, const float *P32,
                              double *w) {
    for (int k = 0; k < n; ++k) or_closure_weights(q + 5 * k, head, method, P64, P32, w + 3 * k);
}

void or_reconstruct_h_batch(const double *q, int n, int head, int method, const double *P64, const float *P32,
                            double h, double *out) {
    for (int k = 0; k < n; ++k) out[k] = or_reconstruct_h(q + 5 * k, head, method, P64, P32, h);
}

void or_reconstruct_batch(const double *q, int n, int head, int method, const double *P64, const float *P32,
                          double *out) {
    for (int k = 0; k < n; ++k) out[k] = or_reconstruct(q + 5 * k, head, method, P64, P32);
}

void or_mlp_ratios_batch(const double *x, int n, int prec, const double *P64, const float *P32, double *r) {
    for (int k = 0; k < n; ++k) {
        if (prec == OR_METHOD_SR64) {
            or_mlp_ratios_f64(x + 5 * k, P64, r + 3 * k);
        } else {
            float xf[5], o[3];
            for (int i = 0; i < 5; ++i) xf[i] = (float)x[5 * k + i];
            if (prec == OR_METHOD_SR32) or_mlp_ratios_f32(xf, P32, o); else or_mlp_ratios_bf16(xf, P32, o);
            for (int i = 0; i < 3; ++i) r[3 * k + i] = o[i];
        }
    }
}

/* ------------------------------------------------------------------------------------------ */
/* 2D Euler WENO7 (JS, Z, SR) with Shu's fourth-order TVD RK (weno7_point_rk4_shu/point_rk4.py:150-616, */
/* weno7_external_clean/warp_weno7_ader4_helpers_classical_only.py:557-855, 2147-2202).              */
/* Padded arrays [ny+8][nx+8][4], ghost width 4, filled in place before each right-hand side.        */
/* ------------------------------------------------------------------------------------------ */
#define G7 4

static void w7_beta(const double *q, double *b) { /* classical_only.py:558-563 */
    double q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3], q4 = q[4], q5 = q[5], q6 = q[6];
    b[3] = 2107.0*q3*q3 - 9402.0*q4*q3 + 7042.0*q3*q5 - 1854.0*q3*q6 - 17246.0*q4*q5 - 3882.0*q5*q6 + 11003.0*q4*q4 + 7043.0*q5*q5 + 547.0*q6*q6 + 4642.0*q4*q6;
    b[2] = 267.0*q5*q5 - 1642.0*q5*q4 + 1602.0*q5*q3 - 494.0*q5*q2 - 2522.0*q3*q2 + 3443.0*q3*q3 + 547.0*q2*q2 - 5966.0*q4*q3 + 2843.0*q4*q4 + 1922.0*q4*q2;
    b[1] = 267.0*q1*q1 - 494.0*q4*q1 - 1642.0*q2*q1 + 1602.0*q3*q1 - 5966.0*q3*q2 + 3443.0*q3*q3 - 2522.0*q4*q3 + 2843.0*q2*q2 + 547.0*q4*q4 + 1922.0*q4*q2;
    b[0] = 2107.0*q3*q3 + 7042.0*q3*q1 - 1854.0*q3*q0 - 9402.0*q3*q2 - 17246.0*q2*q1 + 4642.0*q2*q0 + 547.0*q0*q0 - 3882.0*q1*q0 + 11003.0*q2*q2 + 7043.0*q1*q1;
}

static double w7_face_cand(int loc, double a, double b, double c, double d) { /* stencil_weno7, dorder 0 */
    if (loc == 5) return 25.0/12.0*a - 23.0/12.0*b + 13.0/12.0*c - 1.0/4.0*d;
    if (loc == 4) return 1.0/4.0*a + 13.0/12.0*b - 5.0/12.0*c + 1.0/12.0*d;
    if (loc == 3) return -1.0/12.0*a + 7.0/12.0*b + 7.0/12.0*c - 1.0/12.0*d;
    if (loc == 2) return 1.0/12.0*a - 5.0/12.0*b + 13.0/12.0*c + 1.0/4.0*d;
    return -1.0/4.0*a + 13.0/12.0*b - 23.0/12.0*c + 25.0/12.0*d;
}

static double w7_gauss_cand(int loc, double a, double b, double c, double d) { /* stencil_weno7_2gauss */
    double s = sqrt(3.0);
    switch (loc) {
    case 1: return (-11.0*s/216.0)*a + (17.0*s/72.0)*b - (35.0*s/72.0)*c + ((65.0*s + 216.0)/216.0)*d;
    case 2: return (7.0*s/216.0)*a - (13.0*s/72.0)*b + ((7.0*s + 72.0)/72.0)*c + (11.0*s/216.0)*d;
    case 3: return (-11.0*s/216.0)*a + ((72.0 - 7.0*s)/72.0)*b + (13.0*s/72.0)*c - (7.0*s/216.0)*d;
    case 4: return ((216.0 - 65.0*s)/216.0)*a + (35.0*s/72.0)*b - (17.0*s/72.0)*c + (11.0*s/216.0)*d;
    case 5: return (11.0*s/216.0)*a - (17.0*s/72.0)*b + (35.0*s/72.0)*c + ((216.0 - 65.0*s)/216.0)*d;
    case 6: return (-7.0*s/216.0)*a + (13.0*s/72.0)*b + ((72.0 - 7.0*s)/72.0)*c - (11.0*s/216.0)*d;
    case 7: return (11.0*s/216.0)*a + ((7.0*s + 72.0)/72.0)*b - (13.0*s/72.0)*c + (7.0*s/216.0)*d;
    default: return ((65.0*s + 216.0)/216.0)*a - (35.0*s/72.0)*b + (17.0*s/72.0)*c - (11.0*s/216.0)*d;
    }
}

static double w7_js_combine(const double *q, const double *s, const double *d) { /* weno7_lr_scalar */
    double b[4];
    w7_beta(q, b);
    double r0 = 1.0 / (1.0e-6 + b[0]), r1 = 1.0 / (1.0e-6 + b[1]), r2 = 1.0 / (1.0e-6 + b[2]), r3 = 1.0 / (1.0e-6 + b[3]);
    double a0 = d[0] * r0 * r0, a1 = d[1] * r1 * r1, a2 = d[2] * r2 * r2, a3 = d[3] * r3 * r3;
    double asum = a0 + a1 + a2 + a3;
    return (a0 * s[0] + a1 * s[1] + a2 * s[2] + a3 * s[3]) / asum;
}

double or_w7_face(const double *q, int lr) {
    double s[4];
    int o = lr == 1 ? 1 : 2;
    for (int k = 0; k < 4; ++k) s[k] = w7_face_cand(o + k, q[k], q[k + 1], q[k + 2], q[k + 3]);
    double d1[4] = {1.0/35.0, 12.0/35.0, 18.0/35.0, 4.0/35.0}, d2[4] = {4.0/35.0, 18.0/35.0, 12.0/35.0, 1.0/35.0};
    return w7_js_combine(q, s, lr == 1 ? d1 : d2);
}

double or_w7_gauss(const double *q, int lr) { /* weno7_gauss_lr_scalar */
    double r3 = sqrt(3.0), s[4], d[4];
    int o = lr == 1 ? 1 : 5;
    for (int k = 0; k < 4; ++k) s[k] = w7_gauss_cand(o + k, q[k], q[k + 1], q[k + 2], q[k + 3]);
    if (lr == 1) {
        d[0] = 59.0/880.0 - 5.0*r3/16632.0; d[1] = 381.0/880.0 - 587.0*r3/194040.0;
        d[2] = 587.0*r3/194040.0 + 381.0/880.0; d[3] = 5.0*r3/16632.0 + 59.0/880.0;
    } else {
        d[0] = 5.0*r3/16632.0 + 59.0/880.0; d[1] = 587.0*r3/194040.0 + 381.0/880.0;
        d[2] = 381.0/880.0 - 587.0*r3/194040.0; d[3] = 59.0/880.0 - 5.0*r3/16632.0;
    }
    return w7_js_combine(q, s, d);
}

/* Betas of the WENO-Z module (weno7_helpers_z.py:557-588): the same quadratic forms (with the common factor
 * 240) written as a sum of squares, non-negative in floating point. */
static void w7_beta_sq(const double *q, double *b) {
    double q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3], q4 = q[4], q5 = q[5], q6 = q[6];
    double c0 = 20.0 / 3.0, c1 = 260.0, c2 = 781.0 / 3.0;
    double a00 = -2.0*q0 + 9.0*q1 - 18.0*q2 + 11.0*q3, a01 = -q0 + 4.0*q1 - 5.0*q2 + 2.0*q3, a02 = -q0 + 3.0*q1 - 3.0*q2 + q3;
    b[0] = c0*a00*a00 + c1*a01*a01 + c2*a02*a02;
    double a10 = q1 - 6.0*q2 + 3.0*q3 + 2.0*q4, a11 = q2 - 2.0*q3 + q4, a12 = -q1 + 3.0*q2 - 3.0*q3 + q4;
    b[1] = c0*a10*a10 + c1*a11*a11 + c2*a12*a12;
    double a20 = -2.0*q2 - 3.0*q3 + 6.0*q4 - q5, a21 = q2 - 2.0*q3 + q4, a22 = -q2 + 3.0*q3 - 3.0*q4 + q5;
    b[2] = c0*a20*a20 + c1*a21*a21 + c2*a22*a22;
    double a30 = -11.0*q3 + 18.0*q4 - 9.0*q5 + 2.0*q6, a31 = 2.0*q3 - 5.0*q4 + 4.0*q5 - q6, a32 = -q3 + 3.0*q4 - 3.0*q5 + q6;
    b[3] = c0*a30*a30 + c1*a31*a31 + c2*a32*a32;
}

/* WENO-Z weights of the WENO7 path, weight_kind 1 (weno_z_borges_p2_results/weno7_helpers_z.py:900-957):
 * betas / 240, tau = |-b0 - 3 b1 + 3 b2 + b3|, alpha = d (1 + (tau / (b + h^3))^3), value = sum (alpha/sum) s. */
static double w7_z_combine(const double *q, const double *s, const double *d, double h) {
    double bb[4];
    w7_beta_sq(q, bb);
    double inv240 = 1.0 / 240.0, eps = h * h * h;
    double b0 = bb[0] * inv240, b1 = bb[1] * inv240, b2 = bb[2] * inv240, b3 = bb[3] * inv240;
    double tau = fabs(-b0 - 3.0 * b1 + 3.0 * b2 + b3);
    double r0 = tau / (b0 + eps), r1 = tau / (b1 + eps), r2 = tau / (b2 + eps), r3 = tau / (b3 + eps);
    double a0 = d[0] * (1.0 + r0 * r0 * r0), a1 = d[1] * (1.0 + r1 * r1 * r1), a2 = d[2] * (1.0 + r2 * r2 * r2),
           a3 = d[3] * (1.0 + r3 * r3 * r3);
    double asum = a0 + a1 + a2 + a3;
    return a0 / asum * s[0] + a1 / asum * s[1] + a2 / asum * s[2] + a3 / asum * s[3];
}

double or_w7z_face(const double *q, int lr, double h) { /* weno7_lr_scalar_normalized */
    double s[4];
    int o = lr == 1 ? 1 : 2;
    for (int k = 0; k < 4; ++k) s[k] = w7_face_cand(o + k, q[k], q[k + 1], q[k + 2], q[k + 3]);
    double d1[4] = {1.0/35.0, 12.0/35.0, 18.0/35.0, 4.0/35.0}, d2[4] = {4.0/35.0, 18.0/35.0, 12.0/35.0, 1.0/35.0};
    return w7_z_combine(q, s, lr == 1 ? d1 : d2, h);
}

double or_w7z_gauss(const double *q, int lr, double h) { /* weno7_gauss_lr_scalar_normalized */
    double r3 = sqrt(3.0), s[4], d[4];
    int o = lr == 1 ? 1 : 5;
    for (int k = 0; k < 4; ++k) s[k] = w7_gauss_cand(o + k, q[k], q[k + 1], q[k + 2], q[k + 3]);
    if (lr == 1) {
        d[0] = 59.0/880.0 - 5.0*r3/16632.0; d[1] = 381.0/880.0 - 587.0*r3/194040.0;
        d[2] = 381.0/880.0 + 587.0*r3/194040.0; d[3] = 59.0/880.0 + 5.0*r3/16632.0;
    } else {
        d[0] = 59.0/880.0 + 5.0*r3/16632.0; d[1] = 381.0/880.0 + 587.0*r3/194040.0;
        d[2] = 381.0/880.0 - 587.0*r3/194040.0; d[3] = 59.0/880.0 - 5.0*r3/16632.0;
    }
    return w7_z_combine(q, s, d, h);
}

/* WENO7-SR: betas from the reflection-symmetric closure, evaluated by torch in the reference
 * (teacherfree_lab_weno7_rk4_distance_balanced_fast/warp_sod/beta_provider.py:27-33, 164-219 and
 * weno7_core.py:139-212, 266-324: features, MLP 6 -> 24 -> 16 -> 16 -> 4 with swish, 6 tanh(raw/6), softmax,
 * averaged with the output of the reflected features; beta = 4 ratio, all ones on a plateau), then consumed by
 * the Warp reconstruction (warp_sod/warp_weno7_external_overwrite_fullall.py:67-143: alpha = d / (beta + 1e-12)^2,
 * w = alpha / max(sum, 1e-300)). The lr = 2 face and the second Gauss point take flip(beta(flip(q))). */
#define W7_H1 24
#define W7_H2 16
#define W7_H3 16
#define W7_NPARAM (6 * W7_H1 + W7_H1 + W7_H1 * W7_H2 + W7_H2 + W7_H2 * W7_H3 + W7_H3 + W7_H3 * 4 + 4)

static void w7sr_raw(const double *P, const double *f, double *out) { /* raw_forward, weno7_core.py:311-318 */
    const double *w1 = P, *b1 = w1 + 6 * W7_H1, *w2 = b1 + W7_H1, *b2 = w2 + W7_H1 * W7_H2, *w3 = b2 + W7_H2;
    const double *b3 = w3 + W7_H2 * W7_H3, *w4 = b3 + W7_H3, *b4 = w4 + W7_H3 * 4;
    double h1[W7_H1], h2[W7_H2], h3[W7_H3], z[4];
    for (int o = 0; o < W7_H1; ++o) {
        double a = 0.0;
        for (int k = 0; k < 6; ++k) a += f[k] * w1[k * W7_H1 + o];
        a += b1[o];
        h1[o] = a * (1.0 / (1.0 + exp(-a)));
    }
    for (int o = 0; o < W7_H2; ++o) {
        double a = 0.0;
        for (int k = 0; k < W7_H1; ++k) a += h1[k] * w2[k * W7_H2 + o];
        a += b2[o];
        h2[o] = a * (1.0 / (1.0 + exp(-a)));
    }
    for (int o = 0; o < W7_H3; ++o) {
        double a = 0.0;
        for (int k = 0; k < W7_H2; ++k) a += h2[k] * w3[k * W7_H3 + o];
        a += b3[o];
        h3[o] = a * (1.0 / (1.0 + exp(-a)));
    }
    double m = -INFINITY, sum = 0.0;
    for (int o = 0; o < 4; ++o) {
        double a = 0.0;
        for (int k = 0; k < W7_H3; ++k) a += h3[k] * w4[k * 4 + o];
        a += b4[o];
        z[o] = 6.0 * tanh(a / 6.0);
        if (z[o] > m) m = z[o];
    }
    for (int o = 0; o < 4; ++o) {
        z[o] = exp(z[o] - m);
        sum += z[o];
    }
    for (int o = 0; o < 4; ++o) out[o] = z[o] / sum;
}

/* _mlp_beta of the beta provider on one 7-point stencil */
void or_w7sr_beta(const double *q, const double *P, double *beta) {
    double delta[4], dmax, qs = 1.0, g = 0.0, f[6], fr[6], ra[4], rb[4];
    double fm[4][3] = {
        {-2.0*q[0] + 9.0*q[1] - 18.0*q[2] + 11.0*q[3], -q[0] + 4.0*q[1] - 5.0*q[2] + 2.0*q[3], -q[0] + 3.0*q[1] - 3.0*q[2] + q[3]},
        {q[1] - 6.0*q[2] + 3.0*q[3] + 2.0*q[4], q[2] - 2.0*q[3] + q[4], -q[1] + 3.0*q[2] - 3.0*q[3] + q[4]},
        {-2.0*q[2] - 3.0*q[3] + 6.0*q[4] - q[5], q[2] - 2.0*q[3] + q[4], -q[2] + 3.0*q[3] - 3.0*q[4] + q[5]},
        {-11.0*q[3] + 18.0*q[4] - 9.0*q[5] + 2.0*q[6], 2.0*q[3] - 5.0*q[4] + 4.0*q[5] - q[6], -q[3] + 3.0*q[4] - 3.0*q[5] + q[6]}};
    for (int k = 0; k < 4; ++k)
        delta[k] = fabs(fm[k][0]) * (1.0 / 36.0) + fabs(fm[k][1]) * (13.0 / 12.0) + fabs(fm[k][2]) * (781.0 / 720.0);
    dmax = fmax(fmax(delta[0], delta[1]), fmax(delta[2], delta[3]));
    for (int k = 0; k < 7; ++k) qs = fmax(qs, fabs(q[k]));
    if (dmax <= 1.0e-13 * qs) { /* plateau_mask */
        for (int k = 0; k < 4; ++k) beta[k] = 1.0;
        return;
    }
    for (int k = 0; k < 4; ++k) f[k] = delta[k] / fmax(dmax, 1.0e-15);
    for (int k = 0; k < 5; ++k) {
        double d2 = q[k] - 2.0 * q[k + 1] + q[k + 2];
        g = fmax(g, fabs(d2) / (fabs(q[k + 1] - q[k]) + fabs(q[k + 2] - q[k + 1]) + 1.0e-15));
    }
    f[4] = fmin(fmax(g, 0.0), 1.0);
    f[5] = fmin(fmax((log10(fmax(dmax / qs, 1.0e-30)) + 16.0) / 16.0, 0.0), 1.0);
    for (int k = 0; k < 4; ++k) fr[k] = f[3 - k];
    fr[4] = f[4];
    fr[5] = f[5];
    w7sr_raw(P, f, ra);
    w7sr_raw(P, fr, rb);
    for (int k = 0; k < 4; ++k) beta[k] = 4.0 * (0.5 * (ra[k] + rb[3 - k]));
}

/* betas of side lr: lr = 1 (and Gauss point 1) the stencil itself, lr = 2 (Gauss point 2) the flipped one */
static void w7sr_side_beta(const double *q, int lr, const double *P, double *beta) {
    if (lr == 1) {
        or_w7sr_beta(q, P, beta);
        return;
    }
    double r[7], b[4];
    for (int k = 0; k < 7; ++k) r[k] = q[6 - k];
    or_w7sr_beta(r, P, b);
    for (int k = 0; k < 4; ++k) beta[k] = b[3 - k];
}

static double w7sr_combine(const double *s, const double *d, const double *beta) { /* _weights_from_beta */
    double ib0 = 1.0 / (beta[0] + 1.0e-12), ib1 = 1.0 / (beta[1] + 1.0e-12), ib2 = 1.0 / (beta[2] + 1.0e-12),
           ib3 = 1.0 / (beta[3] + 1.0e-12);
    double a0 = d[0] * ib0 * ib0, a1 = d[1] * ib1 * ib1, a2 = d[2] * ib2 * ib2, a3 = d[3] * ib3 * ib3;
    double m = fmax(a0 + a1 + a2 + a3, 1.0e-300);
    return a0 / m * s[0] + a1 / m * s[1] + a2 / m * s[2] + a3 / m * s[3];
}

double or_w7sr_face(const double *q, int lr, const double *P) { /* _weno7_lr_scalar_external_beta */
    double s[4], beta[4];
    int o = lr == 1 ? 1 : 2;
    for (int k = 0; k < 4; ++k) s[k] = w7_face_cand(o + k, q[k], q[k + 1], q[k + 2], q[k + 3]);
    double d1[4] = {1.0/35.0, 12.0/35.0, 18.0/35.0, 4.0/35.0}, d2[4] = {4.0/35.0, 18.0/35.0, 12.0/35.0, 1.0/35.0};
    w7sr_side_beta(q, lr, P, beta);
    return w7sr_combine(s, lr == 1 ? d1 : d2, beta);
}

double or_w7sr_gauss(const double *q, int lr, const double *P) { /* _weno7_gauss_lr_scalar_external_beta */
    double r3 = sqrt(3.0), s[4], d[4], beta[4];
    int o = lr == 1 ? 1 : 5;
    for (int k = 0; k < 4; ++k) s[k] = w7_gauss_cand(o + k, q[k], q[k + 1], q[k + 2], q[k + 3]);
    if (lr == 1) {
        d[0] = 59.0/880.0 - 5.0*r3/16632.0; d[1] = 381.0/880.0 - 587.0*r3/194040.0;
        d[2] = 381.0/880.0 + 587.0*r3/194040.0; d[3] = 59.0/880.0 + 5.0*r3/16632.0;
    } else {
        d[0] = 59.0/880.0 + 5.0*r3/16632.0; d[1] = 381.0/880.0 + 587.0*r3/194040.0;
        d[2] = 381.0/880.0 - 587.0*r3/194040.0; d[3] = 59.0/880.0 - 5.0*r3/16632.0;
    }
    w7sr_side_beta(q, lr, P, beta);
    return w7sr_combine(s, d, beta);
}

/* Method of a WENO7 right-hand side: kind 0 JS, 1 Z (eps = h^3 of the reconstruction direction), 2 SR with
 * the FP64 closure P (908 packed parameters). */
enum { W7_JS = 0, W7_Z = 1, W7_SR = 2 };

static double w7_face_m(const double *s, int lr, int kind, double h, const double *P) {
    return kind == W7_Z ? or_w7z_face(s, lr, h) : kind == W7_SR ? or_w7sr_face(s, lr, P) : or_w7_face(s, lr);
}

static double w7_gauss_m(const double *s, int lr, int kind, double h, const double *P) {
    return kind == W7_Z ? or_w7z_gauss(s, lr, h) : kind == W7_SR ? or_w7sr_gauss(s, lr, P) : or_w7_gauss(s, lr);
}

/* weno7_lr_vec_characteristic: Roe(q3, q4) for lr = 1, Roe(q2, q3) for lr = 2 */
static vec4 w7_char_face(const vec4 *q, int lr, int dir, double g, int kind, double h, const double *P) {
    vec4 roe = lr == 2 ? roe_average_state(q[2], q[3], g) : roe_average_state(q[3], q[4], g);
    vec4 c[7], cf;
    for (int k = 0; k < 7; ++k) c[k] = con_to_char(q[k], roe, dir, g);
    for (int f = 0; f < 4; ++f) {
        double s[7];
        for (int k = 0; k < 7; ++k) s[k] = c[k].v[f];
        cf.v[f] = w7_face_m(s, lr, kind, h, P);
    }
    return char_to_con(cf, roe, dir, g);
}

static void w7_fill_bc(double *u, int nx, int ny, int bc) { /* apply_(periodic_)boundary_kernel */
    int nxt = nx + 2 * G7, nyt = ny + 2 * G7;
    for (int j = 0; j < nyt; ++j)
        for (int i = 0; i < nxt; ++i) {
            int si = i, sj = j;
            if (bc == OR_BC_PERIODIC) {
                if (i < G7) si = i + nx; else if (i >= nx + G7) si = i - nx;
                if (j < G7) sj = j + ny; else if (j >= ny + G7) sj = j - ny;
            } else {
                if (i < G7) si = G7; else if (i >= nx + G7) si = nx + G7 - 1;
                if (j < G7) sj = G7; else if (j >= ny + G7) sj = ny + G7 - 1;
            }
            if (si != i || sj != j) store4(u, nxt, j, i, load4(u, nxt, sj, si));
        }
}

/* compute_rhs (point_rk4.py:435-511; compute_rhs_mlp, warp_sod/point_rk4_mlp.py:198-277, for kind 2): rhs
 * interior [ny][nx][4]. src's ghost cells are filled in place. Returns 0, or -1 on allocation failure. */
int or_w7_rhs(double *src, double *rhs, int nx, int ny, double dx, double dy, double g, int bc, int reverse, int kind,
              const double *P) {
    int nxt = nx + 2 * G7, nyt = ny + 2 * G7;
    size_t np = (size_t)nxt * nyt * 4;
    double *xl = calloc(np, 8), *xr = calloc(np, 8), *yl = calloc(np, 8), *yr = calloc(np, 8);
    double *f1 = calloc(np, 8), *f2 = calloc(np, 8), *h1 = calloc(np, 8), *h2 = calloc(np, 8);
    int rc = 0;
    if (!xl || !xr || !yl || !yr || !f1 || !f2 || !h1 || !h2) { rc = -1; goto done; }
    w7_fill_bc(src, nx, ny, bc);
#pragma omp parallel for schedule(dynamic, 1)
    for (int j = 0; j < ny + 8; ++j)
        for (int i = 0; i < nx + 2; ++i) {
            vec4 q[7];
            for (int k = 0; k < 7; ++k) q[k] = load4(src, nxt, j, i + k);
            store4(xl, nxt, j, i, w7_char_face(q, 2, 1, g, kind, dx, P));
            store4(xr, nxt, j, i, w7_char_face(q, 1, 1, g, kind, dx, P));
        }
#pragma omp parallel for schedule(dynamic, 1)
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx + 1; ++i)
            for (int loca = 1; loca <= 2; ++loca) {
                vec4 sl, sr;
                for (int comp = 0; comp < 4; ++comp) {
                    double a[7], b[7];
                    for (int k = 0; k < 7; ++k) {
                        a[k] = xr[((size_t)(j + 1 + k) * nxt + i) * 4 + comp];
                        b[k] = xl[((size_t)(j + 1 + k) * nxt + i + 1) * 4 + comp];
                    }
                    sl.v[comp] = w7_gauss_m(a, loca, kind, dy, P);
                    sr.v[comp] = w7_gauss_m(b, loca, kind, dy, P);
                }
                vec4 f = reverse ? or_hllc_flux(sr, sl, 1, g) : or_hllc_flux(sl, sr, 1, g);
                store4(loca == 1 ? f1 : f2, nxt, j, i, f);
            }
#pragma omp parallel for schedule(dynamic, 1)
    for (int j = 0; j < ny + 2; ++j)
        for (int i = 0; i < nx + 8; ++i) {
            vec4 q[7];
            for (int k = 0; k < 7; ++k) q[k] = load4(src, nxt, j + k, i);
            store4(yl, nxt, j, i, w7_char_face(q, 2, 2, g, kind, dy, P));
            store4(yr, nxt, j, i, w7_char_face(q, 1, 2, g, kind, dy, P));
        }
#pragma omp parallel for schedule(dynamic, 1)
    for (int j = 0; j < ny + 1; ++j)
        for (int i = 0; i < nx; ++i)
            for (int loca = 1; loca <= 2; ++loca) {
                vec4 sl, sr;
                for (int comp = 0; comp < 4; ++comp) {
                    double a[7], b[7];
                    for (int k = 0; k < 7; ++k) {
                        a[k] = yr[((size_t)j * nxt + i + 1 + k) * 4 + comp];
                        b[k] = yl[((size_t)(j + 1) * nxt + i + 1 + k) * 4 + comp];
                    }
                    sl.v[comp] = w7_gauss_m(a, loca, kind, dx, P);
                    sr.v[comp] = w7_gauss_m(b, loca, kind, dx, P);
                }
                vec4 f = reverse ? or_hllc_flux(sr, sl, 2, g) : or_hllc_flux(sl, sr, 2, g);
                store4(loca == 1 ? h1 : h2, nxt, j, i, f);
            }
    {
        double inv_dx = 1.0 / dx, inv_dy = 1.0 / dy;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                for (int comp = 0; comp < 4; ++comp) {
#define A7(a, jy, ix) (a)[((size_t)(jy) * nxt + (ix)) * 4 + comp]
                    double fxl = A7(f1, j, i) + A7(f2, j, i), fxr = A7(f1, j, i + 1) + A7(f2, j, i + 1);
                    double fyb = A7(h1, j, i) + A7(h2, j, i), fyt = A7(h1, j + 1, i) + A7(h2, j + 1, i);
#undef A7
                    rhs[((size_t)j * nx + i) * 4 + comp] = -0.5 * (fxr - fxl) * inv_dx - 0.5 * (fyt - fyb) * inv_dy;
                }
    }
done:
    free(xl); free(xr); free(yl); free(yr); free(f1); free(f2); free(h1); free(h2);
    return rc;
}

static double w7_max_speed(const double *u, int nx, int ny, double g) {
    double m = 0.0;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const double *q = u + ((size_t)(j + G7) * (nx + 2 * G7) + i + G7) * 4;
            double rho = fmax(q[0], 1.0e-15), vx = q[1] / rho, vy = q[2] / rho;
            double p = fmax((g - 1.0) * (q[3] - 0.5 * rho * (vx * vx + vy * vy)), 1.0e-15);
            double a = sqrt(g * p / rho), s = fmax(fabs(vx) + a, fabs(vy) + a);
            if (s > m) m = s;
        }
    return m;
}

/* run_from_initial (point_rk4.py:568-600) with launch_shu_rk4_step (514-538): u is advanced in place.
 * Returns the step count (dts receives up to max_dts values) or -1 on allocation failure. */
int or_w7_run(double *u, int nx, int ny, double dx, double dy, double g, double cfl, double t_end, int bc, int kind,
              const double *P, int max_steps, double *dts, int max_dts, double *t_out) {
    size_t np = (size_t)(nx + 2 * G7) * (ny + 2 * G7) * 4, ni = (size_t)nx * ny * 4;
    double *u1 = calloc(np, 8), *u2 = calloc(np, 8), *u3 = calloc(np, 8);
    double *r0 = calloc(ni, 8), *rt0 = calloc(ni, 8), *r1 = calloc(ni, 8), *rt1 = calloc(ni, 8),
           *r2 = calloc(ni, 8), *r3 = calloc(ni, 8);
    int nxt = nx + 2 * G7, step = 0;
    double t = 0.0;
    if (!u1 || !u2 || !u3 || !r0 || !rt0 || !r1 || !rt1 || !r2 || !r3) { step = -1; goto done; }
    while (t < t_end && step < max_steps) {
        double ms = w7_max_speed(u, nx, ny, g);
        double dt = ms < 1.0e-15 ? 1.0e10 : cfl * fmin(dx, dy) / ms;
        if (t + dt > t_end) dt = t_end - t;
        if (dt <= 0.0) break;
#define IN7(a, j, i, c) (a)[((size_t)((j) + G7) * nxt + (i) + G7) * 4 + (c)]
#define RI7(a, j, i, c) (a)[((size_t)(j) * nx + (i)) * 4 + (c)]
        if (or_w7_rhs(u, r0, nx, ny, dx, dy, g, bc, 0, kind, P)) { step = -1; goto done; }
        for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) for (int c = 0; c < 4; ++c)
            IN7(u1, j, i, c) = IN7(u, j, i, c) + 0.5 * dt * RI7(r0, j, i, c);
        if (or_w7_rhs(u, rt0, nx, ny, dx, dy, g, bc, 1, kind, P) || or_w7_rhs(u1, r1, nx, ny, dx, dy, g, bc, 0, kind, P)) {
            step = -1; goto done;
        }
        for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) for (int c = 0; c < 4; ++c)
            IN7(u2, j, i, c) = 649.0/1600.0 * IN7(u, j, i, c) - 10890423.0/25193600.0 * dt * RI7(rt0, j, i, c)
                               + 951.0/1600.0 * IN7(u1, j, i, c) + 5000.0/7873.0 * dt * RI7(r1, j, i, c);
        if (or_w7_rhs(u1, rt1, nx, ny, dx, dy, g, bc, 1, kind, P) || or_w7_rhs(u2, r2, nx, ny, dx, dy, g, bc, 0, kind, P)) {
            step = -1; goto done;
        }
        for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) for (int c = 0; c < 4; ++c)
            IN7(u3, j, i, c) = 53989.0/2500000.0 * IN7(u, j, i, c) - 102261.0/5000000.0 * dt * RI7(rt0, j, i, c)
                               + 4806213.0/20000000.0 * IN7(u1, j, i, c) - 5121.0/20000.0 * dt * RI7(rt1, j, i, c)
                               + 23619.0/32000.0 * IN7(u2, j, i, c) + 7873.0/10000.0 * dt * RI7(r2, j, i, c);
        if (or_w7_rhs(u3, r3, nx, ny, dx, dy, g, bc, 0, kind, P)) { step = -1; goto done; }
        for (int j = 0; j < ny; ++j) for (int i = 0; i < nx; ++i) for (int c = 0; c < 4; ++c)
            IN7(u, j, i, c) = 1.0/5.0 * IN7(u, j, i, c) + 1.0/10.0 * dt * RI7(r0, j, i, c)
                              + 6127.0/30000.0 * IN7(u1, j, i, c) + 1.0/6.0 * dt * RI7(r1, j, i, c)
                              + 7873.0/30000.0 * IN7(u2, j, i, c) + 1.0/3.0 * IN7(u3, j, i, c)
                              + 1.0/6.0 * dt * RI7(r3, j, i, c);
#undef IN7
#undef RI7
        t += dt;
        if (dts && step < max_dts) dts[step] = dt;
        ++step;
    }
    if (t_out) *t_out = t;
done:
    free(u1); free(u2); free(u3); free(r0); free(rt0); free(r1); free(rt1); free(r2); free(r3);
    return step;
}
