/*
 * hf_oracle.c -- CPU restatement of Heatflow-MPM's Eulerian air substep.  TEST INFRASTRUCTURE ONLY: this code is the
 * checker for the CUDA library (parity tests, smoke check) and the timed CPU baseline in bench.py.  Nothing in the
 * product imports, links or executes it.
 *
 * Compiled twice from this one source (see Makefile): REAL = float  -> liboracle_f32.so (the fp32 mirror of the
 * reference arithmetic) and REAL = double -> liboracle_f64.so (the all-FP64 oracle of the precision study).
 *
 * Layout and semantics follow the reference exactly (file:line within pietis/Heatflow-MPM):
 *   cells (n,n,n), u (n+1,n,n), v (n,n+1,n), w (n,n,n+1), C order, k fastest           grid.py:184-196, heat.py:178-187
 *   trilinear sample with clamped lattice indices                                      fields.py:5-36
 *   MAC velocity sample, face geometry, midpoint back-trace                             fields.py:68-116
 *   every kernel of the air path, operation by operation in binary32 (no FMA)          grid.py:25-174, heat.py:12-174,
 *                                                                                       solver.py:19-38
 *   stage order, buffer swaps and the pressure-rhs mean subtraction                    solver.py:63-88, grid.py:219-251
 *   Jacobi-PCG with warp.optim.linear.cg semantics (third-party, warp-lang >= 1.7; restated from its published
 *   algorithm): atol = max(tol*||b||, tol, eps^(9/4)); r.r <= atol^2 freezes x on every iteration; iterations run in
 *   pairs; the host-side test (and so the reported count) happens every check_every iterations.
 *
 * Two switches select between the reference's order-dependent arithmetic and the build's deterministic design:
 *   mean_mode    0: sum of the pressure rhs in fp64, rounded once (the CUDA build);
 *                1: numpy float32 pairwise summation, as rhs.numpy().mean() in grid.py:239 (the reference).
 *   scatter_mode 0: every particle weight (binary32, as the reference forms it) is rounded to a 2^-40 fixed-point
 *                   integer and summed exactly, then rounded once to binary32 (the CUDA build: order-free);
 *                1: sequential binary32 adds in particle order (what the reference's atomics give when run serially).
 * CG inner products are accumulated in fp64 over fixed blocks of 4096 entries summed in block order (deterministic for
 * any thread count); alpha and beta are fp64 and applied to the REAL vectors after rounding to REAL.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef REAL
#define REAL float
#endif
#define R(x) ((REAL)(x))

#ifdef _OPENMP
#include <omp.h>
#endif

#define FX_SCALE 1099511627776.0 /* 2^40 */

typedef struct or_scene {
    int32_t n, n_particles;
    int32_t cg_max_iter, buoyancy, heat_maxiter, heat_check_every, grid_check_every, mean_mode, scatter_mode, pad0;
    double h, rho, t_amb, alpha_f_min, cg_tol, kappa_air, kappa_mat, rate, t_cap, g, heat_tol;
    double vol, k_particle, t_sol, t_liq, y_solid, mu_s, mu_l, t_max;
    /* air grid */
    REAL *u, *v, *w, *su, *sv, *sw;
    REAL *ax, *ay, *az, *qx, *qy, *qz, *kx, *ky, *kz, *mx, *my, *mz;
    REAL *p, *rhs, *alpha_s, *diag;
    REAL *st_alpha, *st_kx, *st_ky, *st_kz, *st_mx, *st_my, *st_mz;
    /* heat */
    REAL *T, *T2, *Tw, *kap, *alpha, *tsum, *tfix, *hrhs, *hdiag;
    int32_t *fixed, *src;
    /* particles */
    REAL *pos, *pvel, *ptemp, *pmelt, *pyield, *pvisc;
    /* CG scratch (n^3 each) and fixed-point accumulators (n+1)^3 each, 12 of them */
    REAL *cg_r, *cg_z, *cg_p, *cg_Ap;
    int64_t *acc;
    /* results of the last substep */
    int32_t heat_iters, grid_iters, heat_done, grid_done;
    double heat_res, grid_res, heat_atol, grid_atol, mean;
} or_scene;

/* ------------------------------------------------------------------------------------------------ lattice helpers */
static inline REAL floorR(REAL x) { return sizeof(REAL) == 4 ? (REAL)floorf((float)x) : (REAL)floor((double)x); }
static inline int clampi(int i, int lo, int hi) { return i < lo ? lo : (i > hi ? hi : i); }
static inline REAL minR(REAL a, REAL b) { return a < b ? a : b; }
static inline REAL maxR(REAL a, REAL b) { return a > b ? a : b; }
static inline REAL clampR(REAL x, REAL lo, REAL hi) { return minR(maxR(lo, x), hi); }

/* fields.py:25-36: trilinear sample of a (nx,ny,nz) lattice whose nodes sit at (i + off) h */
static inline REAL sample(const REAL *a, REAL px, REAL py, REAL pz, REAL ox, REAL oy, REAL oz, REAL h, int nx, int ny,
                          int nz) {
    REAL gx = px / h - ox, gy = py / h - oy, gz = pz / h - oz;
    int ix = (int)floorR(gx), iy = (int)floorR(gy), iz = (int)floorR(gz);
    REAL fx = gx - (REAL)ix, fy = gy - (REAL)iy, fz = gz - (REAL)iz;
    REAL s = R(0.0);
    for (int dx = 0; dx < 2; ++dx) {
        int cx = clampi(ix + dx, 0, nx - 1);
        REAL wx = dx ? fx : R(1.0) - fx;
        for (int dy = 0; dy < 2; ++dy) {
            int cy = clampi(iy + dy, 0, ny - 1);
            REAL wy = dy ? fy : R(1.0) - fy;
            for (int dz = 0; dz < 2; ++dz) {
                int cz = clampi(iz + dz, 0, nz - 1);
                REAL wz = dz ? fz : R(1.0) - fz;
                s += wx * wy * wz * a[((size_t)cx * ny + cy) * nz + cz];
            }
        }
    }
    return s;
}

/* fields.py:68-72 */
static inline void sample_velocity(const REAL *u, const REAL *v, const REAL *w, REAL px, REAL py, REAL pz, REAL h, int n,
                                   REAL *o) {
    o[0] = sample(u, px, py, pz, R(0.0), R(0.5), R(0.5), h, n + 1, n, n);
    o[1] = sample(v, px, py, pz, R(0.5), R(0.0), R(0.5), h, n, n + 1, n);
    o[2] = sample(w, px, py, pz, R(0.5), R(0.5), R(0.0), h, n, n, n + 1);
}

/* fields.py:111-116: x - dt u(x - dt/2 u(x)) */
static inline void backtrace(const REAL *u, const REAL *v, const REAL *w, const REAL *x, REAL h, int n, REAL dt, REAL *o) {
    REAL vel[3], y[3];
    sample_velocity(u, v, w, x[0], x[1], x[2], h, n, vel);
    REAL hdt = R(0.5) * dt;
    for (int c = 0; c < 3; ++c) y[c] = x[c] - hdt * vel[c];
    sample_velocity(u, v, w, y[0], y[1], y[2], h, n, vel);
    for (int c = 0; c < 3; ++c) o[c] = x[c] - dt * vel[c];
}

static inline void face_dims(int axis, int n, int *d) {
    d[0] = n + (axis == 0);
    d[1] = n + (axis == 1);
    d[2] = n + (axis == 2);
}

static inline size_t fidx(const int *d, int i, int j, int k) { return ((size_t)i * d[1] + j) * d[2] + k; }

#define CIDX(i, j, k) ((((size_t)(i)) * n + (j)) * n + (k))

/* ------------------------------------------------------------------------------------------------ grid.py kernels */
/* grid.py:25-33 */
void or_advect_face(int n, double h_, double dt_, const REAL *u, const REAL *v, const REAL *w, int axis, const REAL *q,
                    REAL *out) {
    REAL h = R(h_), dt = R(dt_);
    int d[3];
    face_dims(axis, n, d);
    REAL off[3] = {R(0.5), R(0.5), R(0.5)};
    off[axis] = R(0.0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < d[0]; ++i)
        for (int j = 0; j < d[1]; ++j)
            for (int k = 0; k < d[2]; ++k) {
                int idx = axis == 0 ? i : (axis == 1 ? j : k);
                size_t t = fidx(d, i, j, k);
                if (idx == 0 || idx == n) {
                    out[t] = R(0.0);
                    continue;
                }
                REAL x[3]; /* fields.py:75-81 face_position */
                if (axis == 0) { x[0] = (REAL)i * h; x[1] = ((REAL)j + R(0.5)) * h; x[2] = ((REAL)k + R(0.5)) * h; }
                else if (axis == 1) { x[0] = ((REAL)i + R(0.5)) * h; x[1] = (REAL)j * h; x[2] = ((REAL)k + R(0.5)) * h; }
                else { x[0] = ((REAL)i + R(0.5)) * h; x[1] = ((REAL)j + R(0.5)) * h; x[2] = (REAL)k * h; }
                REAL y[3];
                backtrace(u, v, w, x, h, n, dt, y);
                out[t] = sample(q, y[0], y[1], y[2], off[0], off[1], off[2], h, d[0], d[1], d[2]);
            }
}

/* grid.py:36-43 */
void or_buoyancy(int n, double dt_, double g_, double t_amb_, REAL *w, const REAL *T) {
    REAL dt = R(dt_), g = R(g_), t_amb = R(t_amb_);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            for (int k = 1; k < n; ++k) {
                REAL tf = R(0.5) * (T[CIDX(i, j, k - 1)] + T[CIDX(i, j, k)]);
                size_t t = ((size_t)i * n + j) * (n + 1) + k;
                w[t] = w[t] + dt * g * (tf - t_amb) / (t_amb + R(273.15));
            }
}

/* grid.py:46-59 */
void or_face_fraction(int n, const REAL *alpha_s, int axis, double afmin_, REAL *af) {
    REAL afmin = R(afmin_);
    int d[3];
    face_dims(axis, n, d);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < d[0]; ++i)
        for (int j = 0; j < d[1]; ++j)
            for (int k = 0; k < d[2]; ++k) {
                int idx = axis == 0 ? i : (axis == 1 ? j : k);
                size_t t = fidx(d, i, j, k);
                if (idx == 0 || idx == n) {
                    af[t] = R(0.0);
                    continue;
                }
                REAL a;
                if (axis == 0) a = R(0.5) * (alpha_s[CIDX(i - 1, j, k)] + alpha_s[CIDX(i, j, k)]);
                else if (axis == 1) a = R(0.5) * (alpha_s[CIDX(i, j - 1, k)] + alpha_s[CIDX(i, j, k)]);
                else a = R(0.5) * (alpha_s[CIDX(i, j, k - 1)] + alpha_s[CIDX(i, j, k)]);
                af[t] = clampR(R(1.0) - a, afmin, R(1.0));
            }
}

/* grid.py:62-67 */
void or_zero_wall(int n, int axis, REAL *q) {
    int d[3];
    face_dims(axis, n, d);
    for (int i = 0; i < d[0]; ++i)
        for (int j = 0; j < d[1]; ++j)
            for (int k = 0; k < d[2]; ++k) {
                int idx = axis == 0 ? i : (axis == 1 ? j : k);
                if (idx == 0 || idx == n) q[fidx(d, i, j, k)] = R(0.0);
            }
}

/* grid.py:70-79 */
void or_relax(int n, double h_, double dt_, double rho_, double afmin_, int axis, REAL *q, const REAL *kf, const REAL *mf,
              const REAL *af) {
    REAL h = R(h_), dt = R(dt_), rho = R(rho_), afmin = R(afmin_);
    int d[3];
    face_dims(axis, n, d);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < d[0]; ++i)
        for (int j = 0; j < d[1]; ++j)
            for (int k = 0; k < d[2]; ++k) {
                int idx = axis == 0 ? i : (axis == 1 ? j : k);
                if (idx == 0 || idx == n) continue;
                size_t t = fidx(d, i, j, k);
                REAL c = R(1.0) / (rho * maxR(af[t], afmin) * h * h * h);
                q[t] = (q[t] + dt * c * mf[t]) / (R(1.0) + dt * c * kf[t]);
            }
}

/* grid.py:82-91; scale is given in double and rounded like a Python float kernel argument */
void or_divergence_rhs(int n, double h_, double scale_, const REAL *u, const REAL *v, const REAL *w, const REAL *ax,
                       const REAL *ay, const REAL *az, const REAL *qx, const REAL *qy, const REAL *qz, REAL *rhs) {
    REAL h = R(h_), scale = R(scale_);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            for (int k = 0; k < n; ++k) {
                size_t u0 = ((size_t)i * n + j) * n + k, u1 = ((size_t)(i + 1) * n + j) * n + k;
                size_t v0 = ((size_t)i * (n + 1) + j) * n + k, v1 = ((size_t)i * (n + 1) + j + 1) * n + k;
                size_t w0 = ((size_t)i * n + j) * (n + 1) + k, w1 = w0 + 1;
                REAL div = (ax[u1] * u[u1] + qx[u1] - ax[u0] * u[u0] - qx[u0] + ay[v1] * v[v1] + qy[v1] - ay[v0] * v[v0] -
                            qy[v0] + az[w1] * w[w1] + qz[w1] - az[w0] * w[w0] - qz[w0]) /
                           h;
                rhs[CIDX(i, j, k)] = -scale * div;
            }
}

/* grid.py:94-115 */
void or_laplacian(int n, double h_, double alpha_, double beta_, const REAL *p, const REAL *ax, const REAL *ay,
                  const REAL *az, const REAL *y, REAL *out) {
    REAL h = R(h_), alpha = R(alpha_), beta = R(beta_);
    size_t N = (size_t)n * n * n, nn = (size_t)n * n;
#pragma omp parallel for schedule(static)
    for (size_t t = 0; t < N; ++t) {
        int k = (int)(t % n), j = (int)((t / n) % n), i = (int)(t / nn);
        REAL pc = p[t], acc = R(0.0);
        size_t uu = ((size_t)i * n + j) * n + k, vv = ((size_t)i * (n + 1) + j) * n + k, ww = ((size_t)i * n + j) * (n + 1) + k;
        if (i > 0) acc += ax[uu] * (pc - p[t - nn]);
        if (i < n - 1) acc += ax[uu + nn] * (pc - p[t + nn]);
        if (j > 0) acc += ay[vv] * (pc - p[t - n]);
        if (j < n - 1) acc += ay[vv + n] * (pc - p[t + n]);
        if (k > 0) acc += az[ww] * (pc - p[t - 1]);
        if (k < n - 1) acc += az[ww + 1] * (pc - p[t + 1]);
        out[t] = alpha * acc / (h * h) + beta * y[t];
    }
}

/* grid.py:118-137 */
void or_jacobi(int n, double h_, const REAL *ax, const REAL *ay, const REAL *az, REAL *d) {
    REAL h = R(h_);
    size_t N = (size_t)n * n * n, nn = (size_t)n * n;
#pragma omp parallel for schedule(static)
    for (size_t t = 0; t < N; ++t) {
        int k = (int)(t % n), j = (int)((t / n) % n), i = (int)(t / nn);
        size_t uu = ((size_t)i * n + j) * n + k, vv = ((size_t)i * (n + 1) + j) * n + k, ww = ((size_t)i * n + j) * (n + 1) + k;
        REAL s = R(0.0);
        if (i > 0) s += ax[uu];
        if (i < n - 1) s += ax[uu + nn];
        if (j > 0) s += ay[vv];
        if (j < n - 1) s += ay[vv + n];
        if (k > 0) s += az[ww];
        if (k < n - 1) s += az[ww + 1];
        d[t] = (h * h) / maxR(s, R(1.0e-12));
    }
}

/* grid.py:140-153 */
void or_project(int n, double h_, double dtr_, int axis, REAL *q, const REAL *p) {
    REAL h = R(h_), dtr = R(dtr_);
    int d[3];
    face_dims(axis, n, d);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < d[0]; ++i)
        for (int j = 0; j < d[1]; ++j)
            for (int k = 0; k < d[2]; ++k) {
                int idx = axis == 0 ? i : (axis == 1 ? j : k);
                size_t t = fidx(d, i, j, k);
                if (idx == 0 || idx == n) {
                    q[t] = R(0.0);
                    continue;
                }
                REAL gp;
                if (axis == 0) gp = p[CIDX(i, j, k)] - p[CIDX(i - 1, j, k)];
                else if (axis == 1) gp = p[CIDX(i, j, k)] - p[CIDX(i, j - 1, k)];
                else gp = p[CIDX(i, j, k)] - p[CIDX(i, j, k - 1)];
                q[t] = q[t] - dtr * gp / h;
            }
}

/* grid.py:156-162 */
void or_cell_velocity(int n, const REAL *u, const REAL *v, const REAL *w, REAL *out) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            for (int k = 0; k < n; ++k) {
                size_t t = CIDX(i, j, k);
                out[3 * t + 0] = R(0.5) * (u[((size_t)i * n + j) * n + k] + u[((size_t)(i + 1) * n + j) * n + k]);
                out[3 * t + 1] = R(0.5) * (v[((size_t)i * (n + 1) + j) * n + k] + v[((size_t)i * (n + 1) + j + 1) * n + k]);
                out[3 * t + 2] = R(0.5) * (w[((size_t)i * n + j) * (n + 1) + k] + w[((size_t)i * n + j) * (n + 1) + k + 1]);
            }
}

/* ------------------------------------------------------------------------------------------------ heat.py kernels */
/* heat.py:21-28 */
void or_blend(int n, const REAL *T, const REAL *alpha, const REAL *tsum, REAL *out) {
    size_t N = (size_t)n * n * n;
#pragma omp parallel for schedule(static)
    for (size_t t = 0; t < N; ++t) out[t] = alpha[t] > R(0.05) ? tsum[t] / alpha[t] : T[t];
}

/* heat.py:147-151 */
void or_apply_fixed(int n, REAL *T, const int32_t *fixed, const REAL *tfix) {
    size_t N = (size_t)n * n * n;
    for (size_t t = 0; t < N; ++t)
        if (fixed[t] == 1) T[t] = tfix[t];
}

/* heat.py:154-158 */
void or_source(int n, REAL *T, const int32_t *src, double rate_, double t_cap_, double dt_) {
    REAL rate = R(rate_), t_cap = R(t_cap_), dt = R(dt_);
    size_t N = (size_t)n * n * n;
    for (size_t t = 0; t < N; ++t)
        if (src[t] == 1) T[t] = minR(T[t] + rate * dt, maxR(T[t], t_cap));
}

/* heat.py:31-41 */
void or_advect_T(int n, double h_, double dt_, const REAL *T, const REAL *alpha_s, const REAL *u, const REAL *v,
                 const REAL *w, REAL *out) {
    REAL h = R(h_), dt = R(dt_);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            for (int k = 0; k < n; ++k) {
                size_t t = CIDX(i, j, k);
                if (alpha_s[t] > R(0.5)) {
                    out[t] = T[t];
                    continue;
                }
                REAL x[3] = {((REAL)i + R(0.5)) * h, ((REAL)j + R(0.5)) * h, ((REAL)k + R(0.5)) * h}, y[3];
                backtrace(u, v, w, x, h, n, dt, y);
                out[t] = sample(T, y[0], y[1], y[2], R(0.5), R(0.5), R(0.5), h, n, n, n);
            }
}

/* heat.py:44-47 */
void or_conductivity(int n, double kappa_air_, double kappa_mat_, const REAL *alpha, REAL *kap) {
    REAL ka = R(kappa_air_), km = R(kappa_mat_);
    size_t N = (size_t)n * n * n;
#pragma omp parallel for schedule(static)
    for (size_t t = 0; t < N; ++t) kap[t] = ka + (km - ka) * clampR(alpha[t] / R(0.6), R(0.0), R(1.0));
}

/* heat.py:50-52 */
static inline REAL face_kappa(REAL a, REAL b) { return R(2.0) * a * b / (a + b + R(1.0e-12)); }

/* heat.py:55-91 */
static inline REAL neighbour_terms(const REAL *x, const REAL *kap, const int32_t *fixed, const REAL *tfix, size_t t, int i,
                                   int j, int k, int n, int use_fixed) {
    REAL kc = kap[t], acc = R(0.0), xc = x[t];
    static const int DI[6] = {-1, 1, 0, 0, 0, 0}, DJ[6] = {0, 0, -1, 1, 0, 0}, DK[6] = {0, 0, 0, 0, -1, 1};
    for (int s = 0; s < 6; ++s) {
        int ii = i + DI[s], jj = j + DJ[s], kk = k + DK[s];
        if (ii < 0 || jj < 0 || kk < 0 || ii >= n || jj >= n || kk >= n) continue;
        size_t nb = CIDX(ii, jj, kk);
        REAL kf = face_kappa(kc, kap[nb]);
        if (fixed[nb] == 1) {
            if (use_fixed == 1) acc += kf * tfix[nb];
            else acc += kf * xc;
        } else if (use_fixed == 0) {
            acc += kf * (xc - x[nb]);
        }
    }
    return acc;
}

/* heat.py:94-105 */
void or_heat_matvec(int n, double h_, double dt_, double alpha_, double beta_, const REAL *x, const REAL *kap,
                    const int32_t *fixed, const REAL *tfix, const REAL *y, REAL *out) {
    REAL h = R(h_), dt = R(dt_), alpha = R(alpha_), beta = R(beta_);
    size_t N = (size_t)n * n * n, nn = (size_t)n * n;
#pragma omp parallel for schedule(static)
    for (size_t t = 0; t < N; ++t) {
        int k = (int)(t % n), j = (int)((t / n) % n), i = (int)(t / nn);
        if (fixed[t] == 1) {
            out[t] = alpha * x[t] + beta * y[t];
            continue;
        }
        out[t] = alpha * (x[t] + dt / (h * h) * neighbour_terms(x, kap, fixed, tfix, t, i, j, k, n, 0)) + beta * y[t];
    }
}

/* heat.py:108-118 */
void or_heat_rhs(int n, double h_, double dt_, const REAL *T, const REAL *kap, const int32_t *fixed, const REAL *tfix,
                 const REAL *x, REAL *rhs) {
    REAL h = R(h_), dt = R(dt_);
    size_t N = (size_t)n * n * n, nn = (size_t)n * n;
#pragma omp parallel for schedule(static)
    for (size_t t = 0; t < N; ++t) {
        int k = (int)(t % n), j = (int)((t / n) % n), i = (int)(t / nn);
        if (fixed[t] == 1) {
            rhs[t] = tfix[t];
            continue;
        }
        rhs[t] = T[t] + dt / (h * h) * neighbour_terms(x, kap, fixed, tfix, t, i, j, k, n, 1);
    }
}

/* heat.py:121-144 */
void or_heat_diag(int n, double h_, double dt_, const REAL *kap, const int32_t *fixed, REAL *d) {
    REAL h = R(h_), dt = R(dt_);
    size_t N = (size_t)n * n * n, nn = (size_t)n * n;
#pragma omp parallel for schedule(static)
    for (size_t t = 0; t < N; ++t) {
        int k = (int)(t % n), j = (int)((t / n) % n), i = (int)(t / nn);
        if (fixed[t] == 1) {
            d[t] = R(1.0);
            continue;
        }
        REAL kc = kap[t], s = R(0.0);
        if (i > 0) s += face_kappa(kc, kap[t - nn]);
        if (i < n - 1) s += face_kappa(kc, kap[t + nn]);
        if (j > 0) s += face_kappa(kc, kap[t - n]);
        if (j < n - 1) s += face_kappa(kc, kap[t + n]);
        if (k > 0) s += face_kappa(kc, kap[t - 1]);
        if (k < n - 1) s += face_kappa(kc, kap[t + 1]);
        d[t] = R(1.0) / (R(1.0) + dt / (h * h) * s);
    }
}

/* --------------------------------------------------------------------------------------------- particle transfers */
/* fields.py:39-48 scatter with the accumulation chosen by `mode` (see header).  acc: int64 accumulator of the lattice
 * (mode 0) or NULL; a: the REAL lattice (mode 1 adds into it directly). */
static inline void scatter_one(REAL *a, int64_t *acc, REAL px, REAL py, REAL pz, REAL ox, REAL oy, REAL oz, REAL h, int nx,
                               int ny, int nz, REAL val, int mode) {
    REAL gx = px / h - ox, gy = py / h - oy, gz = pz / h - oz;
    int ix = (int)floorR(gx), iy = (int)floorR(gy), iz = (int)floorR(gz);
    REAL fx = gx - (REAL)ix, fy = gy - (REAL)iy, fz = gz - (REAL)iz;
    for (int dx = 0; dx < 2; ++dx) {
        int cx = clampi(ix + dx, 0, nx - 1);
        REAL wx = dx ? fx : R(1.0) - fx;
        for (int dy = 0; dy < 2; ++dy) {
            int cy = clampi(iy + dy, 0, ny - 1);
            REAL wy = dy ? fy : R(1.0) - fy;
            for (int dz = 0; dz < 2; ++dz) {
                int cz = clampi(iz + dz, 0, nz - 1);
                REAL wz = dz ? fz : R(1.0) - fz;
                REAL c = wx * wy * wz * val;
                size_t t = ((size_t)cx * ny + cy) * nz + cz;
                if (mode == 1) a[t] = a[t] + c;
                else acc[t] += (int64_t)llrint((double)c * FX_SCALE);
            }
        }
    }
}

static inline REAL fx_to_real(int64_t v) { return (REAL)((double)v * (1.0 / FX_SCALE)); }

/* solver.py:19-38 and heat.py:12-18 together: particle -> lattice transfers of one substep.
 * outputs (added to, as the reference's atomics add into zeroed arrays):
 *   alpha_s, qx..qz, kx..kz, mx..mz  (AirGrid obstacle fields)  and  alpha, tsum (HeatField).
 * mode 0 needs acc = 12 * (n+1)^3 int64 zero-initialised scratch; it is cleared again on return. */
void or_scatter(int n, int np_, double h_, double vol_, double k0_, const REAL *pos, const REAL *vel, const REAL *temp,
                REAL *alpha_s, REAL *qx, REAL *qy, REAL *qz, REAL *kx, REAL *ky, REAL *kz, REAL *mx, REAL *my, REAL *mz,
                REAL *alpha, REAL *tsum, int mode, int64_t *acc) {
    REAL h = R(h_), vol = R(vol_), k0 = R(k0_);
    size_t M = (size_t)(n + 1) * (n + 1) * (n + 1);
    REAL *dst[12] = {alpha_s, qx, qy, qz, kx, ky, kz, mx, my, mz, alpha, tsum};
    int dims[12][3];
    for (int f = 0; f < 12; ++f) {
        int ax = (f >= 1 && f <= 9) ? (f - 1) % 3 : -1;
        dims[f][0] = n + (ax == 0);
        dims[f][1] = n + (ax == 1);
        dims[f][2] = n + (ax == 2);
    }
    static const REAL OFF[4][3] = {{0.5f, 0.5f, 0.5f}, {0.0f, 0.5f, 0.5f}, {0.5f, 0.0f, 0.5f}, {0.5f, 0.5f, 0.0f}};
    for (int pass = 0; pass < 2; ++pass) {          /* pass 0: k_scatter_particles, pass 1: k_scatter_heat */
        for (int t = 0; t < np_; ++t) {
            REAL px = pos[3 * t], py = pos[3 * t + 1], pz = pos[3 * t + 2];
            REAL frac = vol / (h * h * h);
            if (pass == 0) {
                REAL vp[3] = {vel[3 * t], vel[3 * t + 1], vel[3 * t + 2]};
                REAL vals[10] = {frac, frac * vp[0], frac * vp[1], frac * vp[2], k0, k0, k0, k0 * vp[0], k0 * vp[1], k0 * vp[2]};
                for (int f = 0; f < 10; ++f) {
                    int o = f == 0 ? 0 : 1 + (f - 1) % 3;
                    scatter_one(dst[f], acc ? acc + (size_t)f * M : NULL, px, py, pz, OFF[o][0], OFF[o][1], OFF[o][2], h,
                                dims[f][0], dims[f][1], dims[f][2], vals[f], mode);
                }
            } else {
                scatter_one(dst[10], acc ? acc + 10 * M : NULL, px, py, pz, R(0.5), R(0.5), R(0.5), h, n, n, n, frac, mode);
                scatter_one(dst[11], acc ? acc + 11 * M : NULL, px, py, pz, R(0.5), R(0.5), R(0.5), h, n, n, n, frac * temp[t],
                            mode);
            }
        }
    }
    if (mode == 0) {
        for (int f = 0; f < 12; ++f) {
            size_t cnt = (size_t)dims[f][0] * dims[f][1] * dims[f][2];
            int64_t *a = acc + (size_t)f * M;
            for (size_t t = 0; t < cnt; ++t) {
                if (a[t]) {
                    dst[f][t] = dst[f][t] + fx_to_real(a[t]);
                    a[t] = 0;
                }
            }
        }
    }
}

/* heat.py:161-174 */
void or_particle_update(int n, int np_, double h_, const REAL *pos, const REAL *Tb, const REAL *Ta, double t_sol_,
                        double t_liq_, double y_solid_, double mu_s_, double mu_l_, double t_max_, REAL *temp, REAL *melt,
                        REAL *ys, REAL *visc) {
    REAL h = R(h_), t_sol = R(t_sol_), t_liq = R(t_liq_), y_solid = R(y_solid_), mu_s = R(mu_s_), mu_l = R(mu_l_),
         t_max = R(t_max_);
    for (int t = 0; t < np_; ++t) {
        REAL px = pos[3 * t], py = pos[3 * t + 1], pz = pos[3 * t + 2];
        REAL dT = sample(Ta, px, py, pz, R(0.5), R(0.5), R(0.5), h, n, n, n) -
                  sample(Tb, px, py, pz, R(0.5), R(0.5), R(0.5), h, n, n, n);
        REAL tp = clampR(temp[t] + dT, R(0.0), t_max);
        temp[t] = tp;
        REAL f = clampR((tp - t_sol) / (t_liq - t_sol), R(0.0), R(1.0));
        melt[t] = f;
        ys[t] = y_solid * (R(1.0) - f);
        visc[t] = mu_s * (R(1.0) - f) + mu_l * f;
    }
}

/* ------------------------------------------------------------------------------------------------ reductions */
#define DOT_BLOCK 4096

double or_dot(const REAL *a, const REAL *b, size_t N) {
    size_t nb = (N + DOT_BLOCK - 1) / DOT_BLOCK;
    double *part = (double *)malloc(sizeof(double) * (nb ? nb : 1));
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < nb; ++q) {
        size_t lo = q * DOT_BLOCK, hi = lo + DOT_BLOCK < N ? lo + DOT_BLOCK : N;
        double s = 0.0;
        for (size_t t = lo; t < hi; ++t) s += (double)a[t] * (double)b[t];
        part[q] = s;
    }
    double s = 0.0;
    for (size_t q = 0; q < nb; ++q) s += part[q];
    free(part);
    return s;
}

/* numpy's pairwise summation of a contiguous binary32 array (the float32 accumulation numpy uses for .mean()). */
static REAL pairwise_sum(const REAL *a, size_t n) {
    if (n < 8) {
        REAL res = R(0.0);
        for (size_t i = 0; i < n; ++i) res += a[i];
        return res;
    } else if (n <= 128) {
        REAL r[8], res;
        size_t i;
        for (int j = 0; j < 8; ++j) r[j] = a[j];
        for (i = 8; i < n - (n % 8); i += 8)
            for (int j = 0; j < 8; ++j) r[j] += a[i + j];
        res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
        for (; i < n; ++i) res += a[i];
        return res;
    } else {
        size_t n2 = n / 2;
        n2 -= n2 % 8;
        return pairwise_sum(a, n2) + pairwise_sum(a + n2, n - n2);
    }
}

/* the value subtracted by grid.py:238-241 (mode 1) or the build's fp64 mean rounded once (mode 0) */
double or_mean(const REAL *a, size_t N, int mode) {
    if (mode == 1) {
        REAL s = pairwise_sum(a, N);
        return (double)(s / (REAL)N);
    }
    double s = 0.0;
    for (size_t t = 0; t < N; ++t) s += (double)a[t];
    return (double)(REAL)(s / (double)N);
}

/* --------------------------------------------------------------------------------------------- Jacobi PCG (warp) */
typedef struct {
    int32_t reported, done;
    double res, atol;
} cg_result;

typedef void (*matvec_fn)(const or_scene *s, const REAL *x, const REAL *y, REAL *out, double alpha, double beta, double dt);

static void mv_pressure(const or_scene *s, const REAL *x, const REAL *y, REAL *out, double alpha, double beta, double dt) {
    (void)dt;
    or_laplacian(s->n, s->h, alpha, beta, x, s->ax, s->ay, s->az, y, out);
}

static void mv_heat(const or_scene *s, const REAL *x, const REAL *y, REAL *out, double alpha, double beta, double dt) {
    or_heat_matvec(s->n, s->h, dt, alpha, beta, x, s->kap, s->fixed, s->tfix, y, out);
}

/* warp.optim.linear.cg with M = diag (restated; see header) */
static cg_result pcg(const or_scene *s, matvec_fn A, double dt, const REAL *D, const REAL *b, REAL *x, double tol,
                     int maxiter, int check_every) {
    size_t N = (size_t)s->n * s->n * s->n;
    REAL *r = s->cg_r, *z = s->cg_z, *p = s->cg_p, *Ap = s->cg_Ap;
    cg_result res = {0, 0, 0.0, 0.0};
    double bb = or_dot(b, b, N);
    double atol = tol * sqrt(bb);
    if (atol < tol) atol = tol;
    if (atol < 1.0e-18) atol = 1.0e-18;
    double atol_sq = atol * atol;
    res.atol = atol;
    A(s, x, b, r, -1.0, 1.0, dt);
    double rr = or_dot(r, r, N);
    for (size_t t = 0; t < N; ++t) z[t] = D[t] * r[t];
    double rz = or_dot(r, z, N);
    memset(Ap, 0, sizeof(REAL) * N);
    memcpy(p, z, sizeof(REAL) * N);
    if (rr <= atol_sq) {
        res.res = sqrt(rr);
        return res;
    }
    if (check_every < 2) check_every = 2;
    int cur = 0, done = 0;
    for (;;) {
        for (int half = 0; half < 2; ++half) {
            A(s, p, Ap, Ap, 1.0, 0.0, dt);
            double pAp = or_dot(p, Ap, N);
            int live = rr > atol_sq;
            REAL alpha = live ? (REAL)(rz / pAp) : R(0.0);
#pragma omp parallel for schedule(static)
            for (size_t t = 0; t < N; ++t) {
                x[t] = x[t] + alpha * p[t];
                r[t] = r[t] - alpha * Ap[t];
            }
            rr = or_dot(r, r, N);
#pragma omp parallel for schedule(static)
            for (size_t t = 0; t < N; ++t) z[t] = D[t] * r[t];
            double rz_new = or_dot(r, z, N);
            REAL beta = rr > atol_sq ? (REAL)(rz_new / rz) : R(0.0);
#pragma omp parallel for schedule(static)
            for (size_t t = 0; t < N; ++t) p[t] = z[t] + beta * p[t];
            rz = rz_new;
            done += live;
        }
        cur += 2;
        if (cur >= maxiter) break;
        if (cur % check_every < 2 && rr <= atol_sq) break;
    }
    res.reported = cur;
    res.done = done;
    res.res = sqrt(rr);
    return res;
}

/* convergence-exact variant used by the CPU baseline: stops at the first iteration with r.r <= atol^2 instead of running
 * the frozen iterations up to the next host check (x is identical; only the reported count differs). */
static int g_exact_stop = 0;
void or_set_exact_stop(int on) { g_exact_stop = on; }

static cg_result pcg_dispatch(const or_scene *s, matvec_fn A, double dt, const REAL *D, const REAL *b, REAL *x, double tol,
                              int maxiter, int check_every) {
    return pcg(s, A, dt, D, b, x, tol, maxiter, g_exact_stop ? 2 : check_every);
}

double or_pcg_pressure(or_scene *s, double tol, int maxiter, int check_every, int32_t *iters) {
    size_t N = (size_t)s->n * s->n * s->n;
    or_jacobi(s->n, s->h, s->ax, s->ay, s->az, s->diag);
    (void)N;
    cg_result r = pcg(s, mv_pressure, 0.0, s->diag, s->rhs, s->p, tol, maxiter, check_every);
    iters[0] = r.reported;
    iters[1] = r.done;
    return r.res;
}

/* ------------------------------------------------------------------------------------------------ whole substep */
static void add_into(REAL *a, const REAL *b, size_t cnt) {
    for (size_t t = 0; t < cnt; ++t) a[t] = a[t] + b[t];
}

#define SWAP(a, b)       \
    do {                 \
        REAL *tmp_ = (a); \
        (a) = (b);       \
        (b) = tmp_;      \
    } while (0)

/* solver.py:63-88 (the MPM step is the caller's) */
void or_substep(or_scene *s, double dt_) {
    int n = s->n;
    size_t N = (size_t)n * n * n, NU = (size_t)(n + 1) * n * n;
    /* grid.py:202-204 and solver.py:67-68 */
    REAL *clr[12] = {s->alpha_s, s->qx, s->qy, s->qz, s->kx, s->ky, s->kz, s->mx, s->my, s->mz, s->alpha, s->tsum};
    for (int f = 0; f < 12; ++f) memset(clr[f], 0, sizeof(REAL) * ((f == 0 || f >= 10) ? N : NU));
    if (s->n_particles > 0)
        or_scatter(n, s->n_particles, s->h, s->vol, s->k_particle, s->pos, s->pvel, s->ptemp, s->alpha_s, s->qx, s->qy,
                   s->qz, s->kx, s->ky, s->kz, s->mx, s->my, s->mz, s->alpha, s->tsum, s->scatter_mode, s->acc);
    /* grid.py:206-213 */
    if (s->st_alpha) {
        add_into(s->alpha_s, s->st_alpha, N);
        add_into(s->kx, s->st_kx, NU);
        add_into(s->ky, s->st_ky, NU);
        add_into(s->kz, s->st_kz, NU);
        add_into(s->mx, s->st_mx, NU);
        add_into(s->my, s->st_my, NU);
        add_into(s->mz, s->st_mz, NU);
    }
    /* solver.py:74-79 */
    or_blend(n, s->T, s->alpha, s->tsum, s->Tw);
    or_apply_fixed(n, s->Tw, s->fixed, s->tfix);
    if (s->rate > 0.0) or_source(n, s->Tw, s->src, s->rate, s->t_cap, dt_);
    or_advect_T(n, s->h, dt_, s->Tw, s->alpha_s, s->u, s->v, s->w, s->T2);
    or_conductivity(n, s->kappa_air, s->kappa_mat, s->alpha_s, s->kap);
    /* heat.py:198-210 */
    or_heat_rhs(n, s->h, dt_, s->T2, s->kap, s->fixed, s->tfix, s->T2, s->hrhs);
    or_heat_diag(n, s->h, dt_, s->kap, s->fixed, s->hdiag);
    cg_result hr = pcg_dispatch(s, mv_heat, dt_, s->hdiag, s->hrhs, s->T2, s->heat_tol, s->heat_maxiter, s->heat_check_every);
    s->heat_iters = hr.reported;
    s->heat_done = hr.done;
    s->heat_res = hr.res;
    s->heat_atol = hr.atol;
    /* solver.py:81-84 */
    if (s->n_particles > 0)
        or_particle_update(n, s->n_particles, s->h, s->pos, s->Tw, s->T2, s->t_sol, s->t_liq, s->y_solid, s->mu_s, s->mu_l,
                           s->t_max, s->ptemp, s->pmelt, s->pyield, s->pvisc);
    SWAP(s->T, s->T2); /* solver.py:85 */
    /* grid.py:219-233 */
    REAL *af[3] = {s->ax, s->ay, s->az}, *qq[3] = {s->qx, s->qy, s->qz};
    for (int a = 0; a < 3; ++a) {
        or_face_fraction(n, s->alpha_s, a, s->alpha_f_min, af[a]);
        or_zero_wall(n, a, qq[a]);
    }
    or_advect_face(n, s->h, dt_, s->u, s->v, s->w, 0, s->u, s->su);
    or_advect_face(n, s->h, dt_, s->u, s->v, s->w, 1, s->v, s->sv);
    or_advect_face(n, s->h, dt_, s->u, s->v, s->w, 2, s->w, s->sw);
    SWAP(s->u, s->su);
    SWAP(s->v, s->sv);
    SWAP(s->w, s->sw);
    if (s->buoyancy) or_buoyancy(n, dt_, s->g, s->t_amb, s->w, s->T);
    REAL *vel[3] = {s->u, s->v, s->w}, *kf[3] = {s->kx, s->ky, s->kz}, *mf[3] = {s->mx, s->my, s->mz};
    for (int a = 0; a < 3; ++a) or_relax(n, s->h, dt_, s->rho, s->alpha_f_min, a, vel[a], kf[a], mf[a], af[a]);
    /* grid.py:235-251; rho/dt and dt/rho are Python floats (double) rounded at the kernel boundary */
    or_divergence_rhs(n, s->h, s->rho / dt_, s->u, s->v, s->w, s->ax, s->ay, s->az, s->qx, s->qy, s->qz, s->rhs);
    double mean = or_mean(s->rhs, N, s->mean_mode);
    s->mean = mean;
    if (mean != 0.0) {
        REAL m = R(mean);
        for (size_t t = 0; t < N; ++t) s->rhs[t] = s->rhs[t] - m;
    }
    or_jacobi(n, s->h, s->ax, s->ay, s->az, s->diag);
    cg_result gr = pcg_dispatch(s, mv_pressure, dt_, s->diag, s->rhs, s->p, s->cg_tol, s->cg_max_iter, s->grid_check_every);
    s->grid_iters = gr.reported;
    s->grid_done = gr.done;
    s->grid_res = gr.res;
    s->grid_atol = gr.atol;
    for (int a = 0; a < 3; ++a) or_project(n, s->h, dt_ / s->rho, a, vel[a], s->p);
}

int or_real_size(void) { return (int)sizeof(REAL); }

int or_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void or_set_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#else
    (void)t;
#endif
}
