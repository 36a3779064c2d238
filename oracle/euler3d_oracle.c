/*
 * CPU oracle for the 3D Euler WENO5 (JS / SR / Z) finite-volume step.
 *
 * TEST INFRASTRUCTURE ONLY. A plain-C restatement of the reference's 3D Warp port, used by the test
 * suite as the parity checker of the CUDA 3D kernels and by bench.py as the timed CPU baseline. The
 * product path never calls it.
 *
 * Reference files (paths inside the reference project, code/snapshot/warp_weno5_3d_rk3/):
 *   kernels.py   9-224   Euler algebra, EVILIN interface state
 *                226-270 Roe average
 *                272-500 left/right eigenvectors for x, y, z
 *                503-672 WENO5-JS face and Gauss-point reconstruction
 *                776-1076 boundary, max speed, normal / transverse / flux kernels
 *                1079-1163 four-point flux difference and the RK stages
 *   mlp_kernels.py, mlp_kernels_f32.py  the SR closure (features of the stencil and of its mirror image,
 *                MLP, reflection average, weights) -- the same closure as the 2D oracle's
 *                or_reconstruct, which this file calls
 *   mlp_normal_scalar.py  the characteristic MLP reconstruction, including the lr = 1 round trip
 *   solver.py    165-329 the order of the sweeps, the four (first_lr, second_lr) flags of the 2x2 Gauss
 *                transverse quadrature, the dt rule and the three RK stages
 *   weno_z_borges_p2_results/weno5_3d_kernels_z.py, weno5_3d_solver_z.py: the same solver with WENO-Z
 *                weights (eps = h^2 of each reconstruction's own direction)
 *
 * Pinned against the reference itself: tests/golden/make_golden_3d.py runs the reference's Warp solver
 * (through a pure-Python stand-in for warp) on a small grid.
 *
 * Additions that the reference does not have (the 3D workload asks for them): an HLLC flux in three
 * dimensions (the 2D HLLC of for_paper_results/solvers/weno5_hllc.py:22-113 with the second tangential
 * velocity carried through the star state), and an inflow state imposed on the x-low ghost cells.
 *
 * Layout: padded row-major q[nz+6][ny+6][nx+6][5] doubles, conserved (rho, rho u, rho v, rho w, E),
 * ghost width 3 (config.py:45-48).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define G3 3

enum { O3_FLUX_EVILIN = 0, O3_FLUX_HLLC = 1 };

typedef struct { double v[5]; } v5;
typedef struct { double m[5][5]; } m55;

/* from euler2d_oracle.c: the 2D/3D scalar closure; WENO-Z (method 4) takes eps = h^2 of the reconstruction
 * direction (weno_z_borges_p2_results/weno5_3d_kernels_z.py:527-562, 673-706) */
double or_reconstruct_h(const double q[5], int head, int method, const double *P64, const float *P32, double h);

static const double GAMMA3 = 1.4;

static v5 con_to_pri5(v5 c) {
    v5 p;
    p.v[0] = c.v[0];
    p.v[1] = c.v[1] / c.v[0];
    p.v[2] = c.v[2] / c.v[0];
    p.v[3] = c.v[3] / c.v[0];
    p.v[4] = (GAMMA3 - 1.0) * (c.v[4] - 0.5 * c.v[0] * (p.v[1] * p.v[1] + p.v[2] * p.v[2] + p.v[3] * p.v[3]));
    return p;
}

static v5 pri_to_con5(v5 p) {
    v5 c;
    c.v[0] = p.v[0];
    c.v[1] = p.v[0] * p.v[1];
    c.v[2] = p.v[0] * p.v[2];
    c.v[3] = p.v[0] * p.v[3];
    c.v[4] = p.v[4] / (GAMMA3 - 1.0) + 0.5 * p.v[0] * (p.v[1] * p.v[1] + p.v[2] * p.v[2] + p.v[3] * p.v[3]);
    return c;
}

static v5 flux_pri5(v5 p, int dir) {
    double rho = p.v[0], u = p.v[1], v = p.v[2], w = p.v[3], pr = p.v[4];
    double e = 0.5 * rho * (u * u + v * v + w * w) + pr / (GAMMA3 - 1.0);
    v5 f;
    if (dir == 1) {
        f.v[0] = rho * u; f.v[1] = rho * u * u + pr; f.v[2] = rho * u * v; f.v[3] = rho * u * w; f.v[4] = u * (pr + e);
    } else if (dir == 2) {
        f.v[0] = rho * v; f.v[1] = rho * u * v; f.v[2] = rho * v * v + pr; f.v[3] = rho * v * w; f.v[4] = v * (pr + e);
    } else {
        f.v[0] = rho * w; f.v[1] = rho * u * w; f.v[2] = rho * v * w; f.v[3] = rho * w * w + pr; f.v[4] = w * (pr + e);
    }
    return f;
}

static v5 clamped_flux5(v5 p, int dir) {
    p.v[0] = fmax(p.v[0], 1.0e-15);
    p.v[4] = fmax(p.v[4], 1.0e-15);
    return flux_pri5(p, dir);
}

static double normal_vel(v5 p, int dir) { return dir == 1 ? p.v[1] : (dir == 2 ? p.v[2] : p.v[3]); }

/* EVILIN interface state (kernels.py:121-223). */
static v5 evilin_state(v5 ul0, v5 ur0, int dir, double dt_dx) {
    const double gamma = GAMMA3, eps = 1.0e-15;
    v5 wl0 = con_to_pri5(ul0), wr0 = con_to_pri5(ur0);
    wl0.v[0] = fmax(wl0.v[0], eps); wl0.v[4] = fmax(wl0.v[4], eps);
    wr0.v[0] = fmax(wr0.v[0], eps); wr0.v[4] = fmax(wr0.v[4], eps);
    double unl0 = normal_vel(wl0, dir), unr0 = normal_vel(wr0, dir);
    double al0 = sqrt(gamma * wl0.v[4] / wl0.v[0]), ar0 = sqrt(gamma * wr0.v[4] / wr0.v[0]);
    double smax = fmax(fabs(unl0) + al0, fabs(unr0) + ar0);
    smax = fmax(smax, eps);
    double dx_dt = 1.0 / dt_dx, courant = smax * dt_dx;
    v5 fl = clamped_flux5(wl0, dir), fr = clamped_flux5(wr0, dir), ulw, ffo, fgf, ulh, urh;
    for (int c = 0; c < 5; ++c) ulw.v[c] = 0.5 * (ul0.v[c] + ur0.v[c]) - 0.5 * dt_dx * (fr.v[c] - fl.v[c]);
    v5 wlw = con_to_pri5(ulw);
    wlw.v[0] = fmax(wlw.v[0], eps); wlw.v[4] = fmax(wlw.v[4], eps);
    v5 flw = clamped_flux5(wlw, dir);
    for (int c = 0; c < 5; ++c) ffo.v[c] = 0.25 * (fl.v[c] + 2.0 * flw.v[c] + fr.v[c] - dx_dt * (ur0.v[c] - ul0.v[c]));
    double theta = (1.0 - courant) / (1.0 + courant);
    for (int c = 0; c < 5; ++c) fgf.v[c] = theta * flw.v[c] + (1.0 - theta) * ffo.v[c];
    for (int c = 0; c < 5; ++c) {
        ulh.v[c] = ul0.v[c] - dt_dx * (fgf.v[c] - fl.v[c]);
        urh.v[c] = ur0.v[c] - dt_dx * (fr.v[c] - fgf.v[c]);
    }
    v5 wl = con_to_pri5(ulh), wr = con_to_pri5(urh);
    wl.v[0] = fmax(wl.v[0], eps); wl.v[4] = fmax(wl.v[4], eps);
    wr.v[0] = fmax(wr.v[0], eps); wr.v[4] = fmax(wr.v[4], eps);
    double rho_bar = fmax(0.5 * (wl.v[0] + wr.v[0]), eps), p_bar = fmax(0.5 * (wl.v[4] + wr.v[4]), eps);
    double a_bar = fmax(sqrt(gamma * p_bar / rho_bar), eps);
    double c1 = rho_bar * a_bar, c2 = rho_bar / a_bar;
    double unle = normal_vel(wl, dir), unre = normal_vel(wr, dir);
    double u_star = 0.5 * (unle + unre) - 0.5 * (wr.v[4] - wl.v[4]) / c1;
    double p_star = 0.5 * (wl.v[4] + wr.v[4]) - 0.5 * (unre - unle) * c1;
    double rho_sl = fmax(wl.v[0] + (unle - u_star) * c2, eps), rho_sr = fmax(wr.v[0] + (u_star - unre) * c2, eps);
    p_star = fmax(p_star, eps);
    double u_bar = 0.5 * (unle + unre);
    double lam1 = u_bar - a_bar, lam2 = u_bar, lam5 = u_bar + a_bar;
    v5 wf = wr;
    int nd = dir;  /* component index of the normal velocity */
    if (lam1 >= 0.0) {
        wf = wl;
    } else if (lam2 >= 0.0) {
        wf = wl; wf.v[0] = rho_sl; wf.v[nd] = u_star; wf.v[4] = p_star;
    } else if (lam5 >= 0.0) {
        wf = wr; wf.v[0] = rho_sr; wf.v[nd] = u_star; wf.v[4] = p_star;
    }
    wf.v[0] = fmax(wf.v[0], eps);
    wf.v[4] = fmax(wf.v[4], eps);
    return pri_to_con5(wf);
}

/* HLLC flux in 3D: Davis speeds, 1e-16 floors, the HLLC5 formulas with the two tangential velocities
 * carried by the star state. */
static double sfloor(double d, double tiny) {
    if (fabs(d) < tiny) return d < 0.0 ? -tiny : tiny;
    return d;
}

static v5 hllc5_flux(v5 ul0, v5 ur0, int dir) {
    const double g = GAMMA3, tiny = 1.0e-16;
    v5 wl = con_to_pri5(ul0), wr = con_to_pri5(ur0);
    double rho_l = fmax(wl.v[0], tiny), rho_r = fmax(wr.v[0], tiny);
    double p_l = fmax(wl.v[4], tiny), p_r = fmax(wr.v[4], tiny);
    double a_l = sqrt(g * p_l / rho_l), a_r = sqrt(g * p_r / rho_r);
    double un_l = normal_vel(wl, dir), un_r = normal_vel(wr, dir);
    double s_l = fmin(un_l - a_l, un_r - a_r), s_r = fmax(un_l + a_l, un_r + a_r);
    v5 f_l = flux_pri5(wl, dir), f_r = flux_pri5(wr, dir);
    if (0.0 <= s_l) return f_l;
    if (0.0 >= s_r) return f_r;
    double denom = sfloor(rho_l * (s_l - un_l) - rho_r * (s_r - un_r), tiny);
    double s_star = (p_r - p_l + rho_l * un_l * (s_l - un_l) - rho_r * un_r * (s_r - un_r)) / denom;
    v5 u_side = ul0, w_side = wl, f_side = f_l;
    double s_side = s_l;
    if (s_star < 0.0) { u_side = ur0; w_side = wr; f_side = f_r; s_side = s_r; }
    double rho = fmax(w_side.v[0], tiny), p = fmax(w_side.v[4], tiny);
    double un = normal_vel(w_side, dir);
    double factor = rho * (s_side - un) / sfloor(s_side - s_star, tiny);
    v5 us;
    us.v[0] = factor;
    for (int c = 1; c <= 3; ++c) us.v[c] = factor * (c == dir ? s_star : w_side.v[c]);
    us.v[4] = factor * ((u_side.v[4] / rho) + (s_star - un) * (s_star + p / (rho * sfloor(s_side - un, tiny))));
    v5 out;
    for (int c = 0; c < 5; ++c) out.v[c] = f_side.v[c] + s_side * (us.v[c] - u_side.v[c]);
    return out;
}

/* Roe-averaged conserved state (kernels.py:226-268). */
static v5 roe5(v5 l, v5 r) {
    const double g = GAMMA3;
    double rl = l.v[0], ul = l.v[1] / rl, vl = l.v[2] / rl, wl = l.v[3] / rl, el = l.v[4];
    double pl = (g - 1.0) * (el - 0.5 * rl * (ul * ul + vl * vl + wl * wl));
    double hl = (el + pl) / rl;
    double rr = r.v[0], ur = r.v[1] / rr, vr = r.v[2] / rr, wr = r.v[3] / rr, er = r.v[4];
    double pr = (g - 1.0) * (er - 0.5 * rr * (ur * ur + vr * vr + wr * wr));
    double hr = (er + pr) / rr;
    double sl = sqrt(rl), sr = sqrt(rr), inv = 1.0 / (sl + sr);
    double u = (sl * ul + sr * ur) * inv, v = (sl * vl + sr * vr) * inv, w = (sl * wl + sr * wr) * inv;
    double h = (sl * hl + sr * hr) * inv, rho = sl * sr;
    double q2 = u * u + v * v + w * w;
    double e = (rho * h + 0.5 * (g - 1.0) * rho * q2) / g;
    v5 out = {{rho, rho * u, rho * v, rho * w, e}};
    return out;
}

/* Left / right eigenvectors of the flux Jacobian in direction dir at a conserved state
 * (kernels.py:272-500): normal velocity component nd, tangential t1 < t2 (x: v, w; y: u, w; z: u, v). */
static void eigen5(v5 s, int dir, m55 *L, m55 *R) {
    const double gm1 = GAMMA3 - 1.0;
    double rho = s.v[0], u = s.v[1] / rho, v = s.v[2] / rho, w = s.v[3] / rho, e = s.v[4];
    double vt = u * u + v * v + w * w;
    double p = gm1 * (e - 0.5 * rho * vt);
    double c = sqrt(GAMMA3 * p / rho), c2 = c * c;
    double h = 0.5 * vt + c2 / gm1;
    double vel[4] = {0.0, u, v, w};
    int nd = dir, t1 = dir == 1 ? 2 : 1, t2 = dir == 3 ? 2 : 3;
    double un = vel[nd], a1 = vel[t1], a2 = vel[t2];
    memset(L, 0, sizeof(*L));
    memset(R, 0, sizeof(*R));
    L->m[0][0] = h + c * (un - c) / gm1;
    L->m[0][nd] = -(un + c / gm1); L->m[0][t1] = -a1; L->m[0][t2] = -a2; L->m[0][4] = 1.0;
    L->m[1][0] = -2.0 * h + 4.0 * c2 / gm1;
    L->m[1][nd] = 2.0 * un; L->m[1][t1] = 2.0 * a1; L->m[1][t2] = 2.0 * a2; L->m[1][4] = -2.0;
    L->m[2][0] = -2.0 * a1 * c2 / gm1; L->m[2][t1] = 2.0 * c2 / gm1;
    L->m[3][0] = -2.0 * a2 * c2 / gm1; L->m[3][t2] = 2.0 * c2 / gm1;
    L->m[4][0] = h - c * (un + c) / gm1;
    L->m[4][nd] = dir == 1 ? -(un - c / gm1) : -un + c / gm1; L->m[4][t1] = -a1; L->m[4][t2] = -a2; L->m[4][4] = 1.0;
    double scale = gm1 / (2.0 * c2);
    for (int r = 0; r < 5; ++r)
        for (int k = 0; k < 5; ++k) L->m[r][k] = L->m[r][k] * scale;
    R->m[0][0] = 1.0; R->m[0][1] = 1.0; R->m[0][4] = 1.0;
    R->m[nd][0] = un - c; R->m[nd][1] = un; R->m[nd][4] = un + c;
    R->m[t1][0] = a1; R->m[t1][1] = a1; R->m[t1][2] = 1.0; R->m[t1][4] = a1;
    R->m[t2][0] = a2; R->m[t2][1] = a2; R->m[t2][3] = 1.0; R->m[t2][4] = a2;
    R->m[4][0] = h - un * c; R->m[4][1] = 0.5 * vt; R->m[4][2] = a1; R->m[4][3] = a2; R->m[4][4] = h + un * c;
}

static v5 matvec(const m55 *M, v5 x) {
    v5 y;
    for (int r = 0; r < 5; ++r) {
        double t = 0.0;
        for (int k = 0; k < 5; ++k) t = t + M->m[r][k] * x.v[k];
        y.v[r] = t;
    }
    return y;
}

/* ------------------------------------------------------------------------------------------ */

typedef struct {
    int nx, ny, nz, method, flux;
    double dx, dy, dz;
    const double *P64;
    const float *P32;
    const double *inflow;  /* 5 conserved values for the x-low ghosts, or NULL (transmissive) */
    int z_halo;            /* z ghost planes given by the caller (a slab of a z-decomposed grid): not filled */
} o3_cfg;

typedef struct {
    double *q0, *nl, *nr, *sl, *sr, *pl, *pr, *fx, *fy, *fz;
} o3_buf;

#define PX(c) ((c)->nx + 2 * G3)
#define PY(c) ((c)->ny + 2 * G3)
#define PZ(c) ((c)->nz + 2 * G3)

static inline size_t at(const o3_cfg *c, int k, int j, int i) { return (((size_t)k * PY(c) + j) * PX(c) + i) * 5; }

static inline v5 ld(const double *a, size_t o) {
    v5 x;
    for (int q = 0; q < 5; ++q) x.v[q] = a[o + q];
    return x;
}

static inline void st(double *a, size_t o, v5 x) {
    for (int q = 0; q < 5; ++q) a[o + q] = x.v[q];
}

/* boundary_x/y/z kernels (kernels.py:776-829), in that order, with the optional inflow state. */
static void boundary(double *q, const o3_cfg *c) {
    int px = PX(c), py = PY(c), pz = PZ(c);
    for (int k = 0; k < pz; ++k)
        for (int j = 0; j < py; ++j) {
            v5 a = ld(q, at(c, k, j, 3)), b = ld(q, at(c, k, j, c->nx + 2));
            if (c->inflow)
                for (int s = 0; s < 5; ++s) a.v[s] = c->inflow[s];
            for (int g = 0; g < 3; ++g) {
                st(q, at(c, k, j, g), a);
                st(q, at(c, k, j, c->nx + 3 + g), b);
            }
        }
    for (int k = 0; k < pz; ++k)
        for (int i = 0; i < px; ++i) {
            v5 a = ld(q, at(c, k, 3, i)), b = ld(q, at(c, k, c->ny + 2, i));
            for (int g = 0; g < 3; ++g) {
                st(q, at(c, k, g, i), a);
                st(q, at(c, k, c->ny + 3 + g, i), b);
            }
        }
    if (c->z_halo) return;
    for (int j = 0; j < py; ++j)
        for (int i = 0; i < px; ++i) {
            v5 a = ld(q, at(c, 3, j, i)), b = ld(q, at(c, c->nz + 2, j, i));
            for (int g = 0; g < 3; ++g) {
                st(q, at(c, g, j, i), a);
                st(q, at(c, c->nz + 3 + g, j, i), b);
            }
        }
}

static double spacing(const o3_cfg *c, int dir) { return dir == 1 ? c->dx : (dir == 2 ? c->dy : c->dz); }

static double recon(const double s[5], int head, int dir, const o3_cfg *c) {
    return or_reconstruct_h(s, head, c->method, c->P64, c->P32, spacing(c, dir));
}

/* Characteristic normal reconstruction of the cell at stencil centre (normal_*_kernel, kernels.py:869-927,
 * and mlp_normal_scalar.py): left = lr 2 (its low face), right = lr 1 (its high face) from the stencil
 * round-tripped through the lr 2 eigenvectors. */
static void normal_cell(const v5 q[5], int dir, const o3_cfg *c, v5 *left, v5 *right) {
    m55 L, R, L1, R1;
    eigen5(roe5(q[1], q[2]), dir, &L, &R);
    v5 ch[5], r[5];
    for (int p = 0; p < 5; ++p) ch[p] = matvec(&L, q[p]);
    v5 cv;
    for (int comp = 0; comp < 5; ++comp) {
        double s[5] = {ch[0].v[comp], ch[1].v[comp], ch[2].v[comp], ch[3].v[comp], ch[4].v[comp]};
        cv.v[comp] = recon(s, 1, dir, c);
    }
    *left = matvec(&R, cv);
    for (int p = 0; p < 5; ++p) r[p] = matvec(&R, ch[p]);
    eigen5(roe5(r[2], r[3]), dir, &L1, &R1);
    for (int p = 0; p < 5; ++p) ch[p] = matvec(&L1, r[p]);
    for (int comp = 0; comp < 5; ++comp) {
        double s[5] = {ch[0].v[comp], ch[1].v[comp], ch[2].v[comp], ch[3].v[comp], ch[4].v[comp]};
        cv.v[comp] = recon(s, 0, dir, c);
    }
    *right = matvec(&R1, cv);
}

static v5 gauss_vec(const v5 q[5], int lr, int dir, const o3_cfg *c) {
    v5 out;
    for (int comp = 0; comp < 5; ++comp) {
        double s[5] = {q[0].v[comp], q[1].v[comp], q[2].v[comp], q[3].v[comp], q[4].v[comp]};
        out.v[comp] = recon(s, lr == 1 ? 2 : 3, dir, c);
    }
    return out;
}

static v5 riemann_flux(v5 ul, v5 ur, int dir, double dt_h, const o3_cfg *c) {
    if (c->flux == O3_FLUX_HLLC) return hllc5_flux(ul, ur, dir);
    return flux_pri5(con_to_pri5(evilin_state(ul, ur, dir, dt_h)), dir);
}

/* One direction's face fluxes, already multiplied by dt/h and summed over the four Gauss points
 * (solver.py:165-283, kernels.py:1015-1076). dir: 1 x, 2 y, 3 z. */
static void sweep(const double *q, int dir, double dt_h, const o3_cfg *c, o3_buf *b, double *flux) {
    int nx = c->nx, ny = c->ny, nz = c->nz, px = PX(c), py = PY(c), pz = PZ(c);
    /* normal: extended ranges (the normal direction covers cells -1 .. n, the others all rows) */
    int kn = dir == 3 ? nz + 2 : pz, jn = dir == 2 ? ny + 2 : py, in = dir == 1 ? nx + 2 : px;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < kn; ++k)
        for (int j = 0; j < jn; ++j)
            for (int i = 0; i < in; ++i) {
                v5 s[5];
                for (int p = 0; p < 5; ++p)
                    s[p] = ld(q, at(c, k + (dir == 3 ? p : 0), j + (dir == 2 ? p : 0), i + (dir == 1 ? p : 0)));
                v5 l, r;
                normal_cell(s, dir, c, &l, &r);
                st(b->nl, at(c, k, j, i), l);
                st(b->nr, at(c, k, j, i), r);
            }
    /* transverse directions: first (a) and second (b) */
    int ta = dir == 1 ? 2 : 1, tb = dir == 3 ? 1 : 3;
    if (dir == 3) { ta = 2; tb = 1; }
    for (int flag = 1; flag <= 4; ++flag) {
        int first_lr = (flag == 1 || flag == 3) ? 1 : 2, second_lr = (flag == 1 || flag == 2) ? 1 : 2;
        /* pass a: along ta over the extent that pass b needs */
        int ka = ta == 3 ? nz : (dir == 3 ? nz + 2 : pz);
        int ja = ta == 2 ? ny : (dir == 2 ? ny + 2 : py);
        int ia = ta == 1 ? nx : (dir == 1 ? nx + 2 : px);
#pragma omp parallel for collapse(2) schedule(static)
        for (int k = 0; k < ka; ++k)
            for (int j = 0; j < ja; ++j)
                for (int i = 0; i < ia; ++i) {
                    v5 sl[5], sr[5];
                    for (int p = 0; p < 5; ++p) {
                        size_t o = at(c, k + (ta == 3 ? p + 1 : 0), j + (ta == 2 ? p + 1 : 0), i + (ta == 1 ? p + 1 : 0));
                        sl[p] = ld(b->nl, o);
                        sr[p] = ld(b->nr, o);
                    }
                    st(b->sl, at(c, k, j, i), gauss_vec(sl, first_lr, ta, c));
                    st(b->sr, at(c, k, j, i), gauss_vec(sr, first_lr, ta, c));
                }
        /* pass b: along tb, over the interior of both transverse directions */
        int kb = dir == 3 ? nz + 2 : nz, jb = dir == 2 ? ny + 2 : ny, ib = dir == 1 ? nx + 2 : nx;
#pragma omp parallel for collapse(2) schedule(static)
        for (int k = 0; k < kb; ++k)
            for (int j = 0; j < jb; ++j)
                for (int i = 0; i < ib; ++i) {
                    v5 sl[5], sr[5];
                    for (int p = 0; p < 5; ++p) {
                        size_t o = at(c, k + (tb == 3 ? p + 1 : 0), j + (tb == 2 ? p + 1 : 0), i + (tb == 1 ? p + 1 : 0));
                        sl[p] = ld(b->sl, o);
                        sr[p] = ld(b->sr, o);
                    }
                    st(b->pl, at(c, k, j, i), gauss_vec(sl, second_lr, tb, c));
                    st(b->pr, at(c, k, j, i), gauss_vec(sr, second_lr, tb, c));
                }
        /* face fluxes: face f between normal-index cells f (right state) and f + 1 (left state) */
        int kf = dir == 3 ? nz + 1 : nz, jf = dir == 2 ? ny + 1 : ny, iff = dir == 1 ? nx + 1 : nx;
#pragma omp parallel for collapse(2) schedule(static)
        for (int k = 0; k < kf; ++k)
            for (int j = 0; j < jf; ++j)
                for (int i = 0; i < iff; ++i) {
                    v5 lft = ld(b->pl, at(c, k + (dir == 3), j + (dir == 2), i + (dir == 1)));
                    v5 rgt = ld(b->pr, at(c, k, j, i));
                    v5 f = riemann_flux(rgt, lft, dir, dt_h, c);
                    size_t o = (((size_t)k * jf + j) * iff + i) * 5;
                    for (int s = 0; s < 5; ++s) {
                        double scaled = f.v[s] * dt_h;
                        flux[o + s] = flag == 1 ? scaled : flux[o + s] + scaled;
                    }
                }
    }
}

static double four_point(double old, double xl, double xr, double yl, double yr, double zl, double zr) {
    return old - 0.25 * (xr - xl) - 0.25 * (yr - yl) - 0.25 * (zr - zl);
}

static void rk_stage(double *q, int stage, double dt, const o3_cfg *c, o3_buf *b) {
    boundary(q, c);
    sweep(q, 1, dt / c->dx, c, b, b->fx);
    sweep(q, 2, dt / c->dy, c, b, b->fy);
    sweep(q, 3, dt / c->dz, c, b, b->fz);
    int nx = c->nx, ny = c->ny, nz = c->nz;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                for (int s = 0; s < 5; ++s) {
                    size_t o = at(c, k + G3, j + G3, i + G3) + s;
                    double fxl = b->fx[(((size_t)k * ny + j) * (nx + 1) + i) * 5 + s];
                    double fxr = b->fx[(((size_t)k * ny + j) * (nx + 1) + i + 1) * 5 + s];
                    double fyl = b->fy[(((size_t)k * (ny + 1) + j) * nx + i) * 5 + s];
                    double fyr = b->fy[(((size_t)k * (ny + 1) + j + 1) * nx + i) * 5 + s];
                    double fzl = b->fz[(((size_t)k * ny + j) * nx + i) * 5 + s];
                    double fzr = b->fz[(((size_t)(k + 1) * ny + j) * nx + i) * 5 + s];
                    double old = q[o];
                    if (stage == 1) {
                        b->q0[o] = old;
                        q[o] = four_point(old, fxl, fxr, fyl, fyr, fzl, fzr);
                    } else if (stage == 2) {
                        double adv = four_point(old, fxl, fxr, fyl, fyr, fzl, fzr);
                        q[o] = (3.0 / 4.0) * b->q0[o] + (1.0 / 4.0) * adv;
                    } else {
                        double adv = four_point(old, fxl, fxr, fyl, fyr, fzl, fzr);
                        q[o] = (1.0 / 3.0) * b->q0[o] + (2.0 / 3.0) * adv;
                    }
                }
}

/* max over the interior of max(|u|, |v|, |w|) + sqrt(1.4 p / rho) (max_speed_kernel, kernels.py:832-845) */
double or_euler3d_max_speed(const double *q, int nx, int ny, int nz) {
    o3_cfg c = {0};
    c.nx = nx; c.ny = ny; c.nz = nz;
    double m = 0.0;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                v5 p = con_to_pri5(ld(q, at(&c, k + G3, j + G3, i + G3)));
                double a = sqrt(GAMMA3 * p.v[4] / p.v[0]);
                double s = fmax(fabs(p.v[1]) + a, fmax(fabs(p.v[2]) + a, fabs(p.v[3]) + a));
                if (s > m) m = s;
            }
    return m;
}

static int alloc_buf(o3_buf *b, const o3_cfg *c) {
    size_t n = (size_t)PX(c) * PY(c) * PZ(c) * 5;
    memset(b, 0, sizeof(*b));
    double **arrs[7] = {&b->q0, &b->nl, &b->nr, &b->sl, &b->sr, &b->pl, &b->pr};
    for (int a = 0; a < 7; ++a) {
        *arrs[a] = (double *)calloc(n, sizeof(double));
        if (!*arrs[a]) return -1;
    }
    b->fx = (double *)calloc((size_t)c->nz * c->ny * (c->nx + 1) * 5, sizeof(double));
    b->fy = (double *)calloc((size_t)c->nz * (c->ny + 1) * c->nx * 5, sizeof(double));
    b->fz = (double *)calloc((size_t)(c->nz + 1) * c->ny * c->nx * 5, sizeof(double));
    return (b->fx && b->fy && b->fz) ? 0 : -1;
}

static void free_buf(o3_buf *b) {
    double *arrs[10] = {b->q0, b->nl, b->nr, b->sl, b->sr, b->pl, b->pr, b->fx, b->fy, b->fz};
    for (int a = 0; a < 10; ++a) free(arrs[a]);
}

/* Advance q (padded, in place) by `steps` steps (Weno5Rk3Solver.advance, solver.py:303-329):
 * dt = cfl min(dx, dy, dz) / max speed (1e10 when the speed is below 1e-15), clipped to t_end.
 * Writes each step's dt to dts (capacity steps) and returns the number of steps taken, or -1. */
int or_euler3d_run(double *q, int nx, int ny, int nz, double dx, double dy, double dz, double cfl, double t_start,
                   double t_end, int steps, int method, int flux, const double *P64, const float *P32,
                   const double *inflow, double *dts, int stage_only) {
    o3_cfg c = {nx, ny, nz, method, flux, dx, dy, dz, P64, P32, inflow};
    o3_buf b;
    if (alloc_buf(&b, &c)) { free_buf(&b); return -1; }
    double t = t_start;
    int taken = 0;
    for (int s = 0; s < steps; ++s) {
        if (t == t_end) break;
        double m = or_euler3d_max_speed(q, nx, ny, nz);
        double raw = m < 1.0e-15 ? 1.0e10 : cfl * fmin(dx, fmin(dy, dz)) / m;
        double dt = raw;
        if (t + dt > t_end) dt = t_end - t;
        t += dt;
        dts[s] = dt;
        rk_stage(q, 1, dt, &c, &b);
        if (stage_only) { ++taken; break; }
        rk_stage(q, 2, dt, &c, &b);
        rk_stage(q, 3, dt, &c, &b);
        ++taken;
    }
    free_buf(&b);
    return taken;
}

/* One RK stage in place (rk_stage) with the stage-start copy in the caller's q0 (padded, kept between the
 * three stages); z_halo: the z ghost planes of q are taken as given. Returns 0, or -1 on allocation failure. */
int or_euler3d_stage(double *q, double *q0, int nx, int ny, int nz, double dx, double dy, double dz, double dt,
                     int stage, int method, int flux, const double *P64, const float *P32, const double *inflow,
                     int z_halo) {
    o3_cfg c = {nx, ny, nz, method, flux, dx, dy, dz, P64, P32, inflow, z_halo};
    o3_buf b;
    if (alloc_buf(&b, &c)) { free_buf(&b); return -1; }
    double *own = b.q0;
    b.q0 = q0;
    rk_stage(q, stage, dt, &c, &b);
    b.q0 = own;
    free_buf(&b);
    return 0;
}

/* Flat wrappers for the flux tests: n interfaces of 5 conserved values each. */
void or_hllc5_batch(const double *ul, const double *ur, int n, int dir, double *out) {
    for (int e = 0; e < n; ++e) {
        v5 a = ld(ul, (size_t)e * 5), b2 = ld(ur, (size_t)e * 5);
        st(out, (size_t)e * 5, hllc5_flux(a, b2, dir));
    }
}

void or_evilin5_batch(const double *ul, const double *ur, int n, int dir, double dt_dx, double *out) {
    for (int e = 0; e < n; ++e) {
        v5 a = ld(ul, (size_t)e * 5), b2 = ld(ur, (size_t)e * 5);
        st(out, (size_t)e * 5, flux_pri5(con_to_pri5(evilin_state(a, b2, dir, dt_dx)), dir));
    }
}
