// hf_cg.cu -- persistent, cooperative Jacobi-preconditioned CG over a batch of scenes.
//
// One launch performs a whole solve (heat.py:198-210 or grid.py:235-251) with the convergence test on the device,
// so no iteration ever waits for the host.  The grid is co-resident (cooperative launch); phases are separated by a
// software grid barrier whose wait is bounded in time (a timeout sets a flag and every block leaves the solve).
//
// Semantics follow warp.optim.linear.cg with M = diag(D) (restated from warp-lang's published algorithm; the package
// is a dependency of the reference, not part of it):
//     r = b - A x,  z = D r,  p = z,  atol = max(tol ||b||, tol, 1e-18)
//     repeat: Ap = A p; alpha = rz / pAp; x += alpha p; r -= alpha Ap; z = D r; beta = rz'/rz; p = z + beta p
//     until r.r <= atol^2 (tested every iteration, which is where the reference's frozen iterations leave x) or maxiter.
// Inner products, alpha and beta are fp64; the vectors stay binary32 and alpha/beta are applied after rounding.
//
// Two grid barriers per iteration: the search-direction update p = z + beta p is not a separate phase -- every block
// recomputes p at the stencil points it reads (its own cells and their neighbours) from z and the previous p, which
// are double-buffered, so the update costs no barrier.
//
// Reductions are deterministic: each 1024-cell chunk produces one fp64 partial in a fixed tree; the block that
// completes a scene's last chunk sums that scene's partials in chunk order (again a fixed tree) and publishes the
// scalars.  The result depends only on the scene, not on the batch it runs in or on the grid size.
#include "hf_device.cuh"
#include "hf_kernels.cuh"

namespace hf {

constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;   // 2 s

__device__ __forceinline__ int uidx_(int n, int i, int j, int k) { return (i * n + j) * n + k; }
__device__ __forceinline__ int vidx_(int n, int i, int j, int k) { return (i * (n + 1) + j) * n + k; }
__device__ __forceinline__ int widx_(int n, int i, int j, int k) { return (i * n + j) * (n + 1) + k; }

// Grid barrier with a bounded wait.  Returns false (in every thread) once any block has timed out.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned& epoch, int* err) {
    ++epoch;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned target = epoch * gridDim.x;
        __threadfence();
        atomicAdd(bar, 1u);
        const unsigned long long t0 = global_timer_ns();
        unsigned spins = 0;
        while (ld_acquire_u32(bar) < target) {
            if (*(volatile int*)err) break;
            if ((++spins & 255u) == 0 && global_timer_ns() - t0 > kBarrierTimeoutNs) {
                atomicExch(err, 1);
                break;
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile int*)err == 0;
}

// Sum of a scene's chunk partials (component q of buffer `buf`) in a fixed tree: threads stride over the scene's chunks in
// order, then block_sum.  Every block that needs the value computes it and obtains the same bits.
template <int K>
__device__ __forceinline__ void scene_sums(const double* __restrict__ buf, int b, int e, const int (&comp)[K],
                                           double (&tot)[K], double* red) {
#pragma unroll
    for (int q = 0; q < K; ++q) tot[q] = 0.0;
    for (int c = b + threadIdx.x; c < e; c += kThreads) {
#pragma unroll
        for (int q = 0; q < K; ++q) tot[q] += buf[3 * c + comp[q]];
    }
    block_sum<K>(tot, red);
}

// Store a chunk's partials (after the block reduction) with plain stores; the next grid barrier publishes them.
template <int K>
__device__ __forceinline__ void put_partials(double* buf, int chunk, double (&part)[K], double* red) {
    block_sum<K>(part, red);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < K; ++q) buf[3 * chunk + q] = part[q];
    }
}

// Search direction at cell t for iteration k: p_k = z + beta p_{k-1} (heat.py/grid.py CG: _cg_kernel_2), or z on the
// first iteration (p_1 = clone(z)).
struct Dir {
    const float* z;
    const float* pold;
    float beta;
    bool first;
    __device__ __forceinline__ float operator()(int t) const {
        return first ? z[t] : __fadd_rn(z[t], __fmul_rn(beta, pold[t]));
    }
};

struct Vec {
    const float* a;
    __device__ __forceinline__ float operator()(int t) const { return a[t]; }
};

// grid.py:94-115 k_laplacian accumulation: sum over the six faces of alpha_f (x_c - x_nb), domain faces skipped
template <class X>
__device__ __forceinline__ float lap_acc(const hf_scene& S, const X& x, float xc, int t, int i, int j, int k) {
    const int n = S.n, nn = n * n;
    float acc = 0.0f;
    if (i > 0) acc = __fadd_rn(acc, __fmul_rn(__ldg(S.ax + uidx_(n, i, j, k)), __fsub_rn(xc, x(t - nn))));
    if (i < n - 1) acc = __fadd_rn(acc, __fmul_rn(__ldg(S.ax + uidx_(n, i + 1, j, k)), __fsub_rn(xc, x(t + nn))));
    if (j > 0) acc = __fadd_rn(acc, __fmul_rn(__ldg(S.ay + vidx_(n, i, j, k)), __fsub_rn(xc, x(t - n))));
    if (j < n - 1) acc = __fadd_rn(acc, __fmul_rn(__ldg(S.ay + vidx_(n, i, j + 1, k)), __fsub_rn(xc, x(t + n))));
    if (k > 0) acc = __fadd_rn(acc, __fmul_rn(__ldg(S.az + widx_(n, i, j, k)), __fsub_rn(xc, x(t - 1))));
    if (k < n - 1) acc = __fadd_rn(acc, __fmul_rn(__ldg(S.az + widx_(n, i, j, k + 1)), __fsub_rn(xc, x(t + 1))));
    return acc;
}

// heat.py:55-91 neighbour_terms with use_fixed = 0; kappa_f from the precomputed face diffusivities
template <class X>
__device__ __forceinline__ float heat_nt(const hf_scene& S, const X& x, float xc, int t, int i, int j, int k) {
    const int n = S.n, nn = n * n;
    const uint8_t* __restrict__ fl = S.cell_flags;
    float acc = 0.0f;
    const int nbr[6] = {t - nn, t + nn, t - n, t + n, t - 1, t + 1};
    const bool in[6] = {i > 0, i < n - 1, j > 0, j < n - 1, k > 0, k < n - 1};
    const int fidx[6] = {uidx_(n, i, j, k), uidx_(n, i + 1, j, k), vidx_(n, i, j, k), vidx_(n, i, j + 1, k),
                         widx_(n, i, j, k), widx_(n, i, j, k + 1)};
    const float* __restrict__ hk[3] = {S.hkx, S.hky, S.hkz};
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        if (!in[s]) continue;
        const int nb = nbr[s];
        const float kf = __ldg(hk[s >> 1] + fidx[s]);
        acc = __fadd_rn(acc, (__ldg(fl + nb) & 1) ? __fmul_rn(kf, xc) : __fmul_rn(kf, __fsub_rn(xc, x(nb))));
    }
    return acc;
}

// heat.py:121-144 k_heat_diag: sum of the in-domain face diffusivities
__device__ __forceinline__ float heat_diag_sum(const hf_scene& S, int i, int j, int k) {
    const int n = S.n;
    float s = 0.0f;
    if (i > 0) s = __fadd_rn(s, S.hkx[uidx_(n, i, j, k)]);
    if (i < n - 1) s = __fadd_rn(s, S.hkx[uidx_(n, i + 1, j, k)]);
    if (j > 0) s = __fadd_rn(s, S.hky[vidx_(n, i, j, k)]);
    if (j < n - 1) s = __fadd_rn(s, S.hky[vidx_(n, i, j + 1, k)]);
    if (k > 0) s = __fadd_rn(s, S.hkz[widx_(n, i, j, k)]);
    if (k < n - 1) s = __fadd_rn(s, S.hkz[widx_(n, i, j, k + 1)]);
    return s;
}

constexpr int kLocalScenes = 32;   // scenes one block may touch (the host checks)

// Per-block copy of a scene's CG scalars.  Every block touching the scene derives them from the same partial sums,
// so all copies agree bit for bit.
struct LocalScene {
    double rz, atol_sq, bb, rr, pAp, mean;
    float alpha, beta;
    int live, iters, maxit, status;
};

template <bool HEAT>
__global__ void __launch_bounds__(kThreads) k_pcg(const hf_scene* __restrict__ scenes, const WorkItem* __restrict__ work,
                                                 int num_chunks, int num_scenes, double dt_d, Workspace ws) {
    __shared__ double red[3 * (kThreads / 32)];
    __shared__ unsigned char s_par[kMaxScenes];
    __shared__ LocalScene loc[kLocalScenes];
    for (int s = threadIdx.x; s < num_scenes; s += kThreads) s_par[s] = (unsigned char)scenes[s].state->parity;
    // contiguous, balanced chunk range of this block and the scenes it touches
    const int c0 = (int)(((long long)num_chunks * blockIdx.x) / gridDim.x);
    const int c1 = (int)(((long long)num_chunks * (blockIdx.x + 1)) / gridDim.x);
    const int s_lo = c0 < c1 ? work[c0].scene : 0;
    const int s_hi = c0 < c1 ? work[c1 - 1].scene : -1;
    __syncthreads();
    unsigned* bar = ws.bar + (HEAT ? 0 : 1);
    unsigned* live_count = ws.live_count + (HEAT ? 0 : 1);
    double* bufA = ws.partials;                       // phase A partials (p.Ap)
    double* bufB = ws.partials + 3 * (size_t)num_chunks;  // prologue / phase B partials (b.b, r.r, r.z)
    unsigned epoch = 0;
    const float dt = (float)dt_d;

    // ---------------------------------------------------------------------------------------- prologue
    // pressure: the mean of the rhs (grid.py:238-241) from the divergence kernel's chunk partials
    for (int s = s_lo; s <= s_hi; ++s) {
        double m[1];
        const int comp[1] = {0};
        if (!HEAT) {
            scene_sums<1>(bufA, ws.chunk_begin[s], ws.chunk_begin[s + 1], comp, m, red);
            const int n = scenes[s].n;
            if (threadIdx.x == 0) loc[s - s_lo].mean = (double)__double2float_rn(m[0] / ((double)n * n * n));
        }
    }
    __syncthreads();
    for (int c = c0; c < c1; ++c) {
        const WorkItem wi = work[c];
        const hf_scene& S = scenes[wi.scene];
        const int n = S.n, N = n * n * n, par = s_par[wi.scene];
        const float h = (float)S.h, hh = __fmul_rn(h, h);
        const float c_dt = __fdiv_rn(dt, hh);
        float* x = HEAT ? S.T[par ^ 1] : S.p;
        const Vec X{x};
        double part[3] = {0.0, 0.0, 0.0};
        const float mean = HEAT ? 0.0f : (float)loc[wi.scene - s_lo].mean;
        for (int m = 0; m < kCellsPerThread; ++m) {
            const int t = wi.first + threadIdx.x + m * kThreads;
            if (t >= N) break;
            int i, j, k;
            cell_ijk(t, n, i, j, k);
            float b, d, r;
            const float xc = x[t];
            if (HEAT) {
                b = S.hrhs[t];
                if (S.cell_flags[t] & 1) {
                    d = 1.0f;
                    r = __fsub_rn(b, xc);
                } else {
                    // heat.py:121-144 k_heat_diag
                    d = __fdiv_rn(1.0f, __fadd_rn(1.0f, __fmul_rn(c_dt, heat_diag_sum(S, i, j, k))));
                    r = __fsub_rn(b, __fadd_rn(xc, __fmul_rn(c_dt, heat_nt(S, X, xc, t, i, j, k))));
                }
                S.hdiag[t] = d;
            } else {
                // grid.py:238-241 mean removal, grid.py:118-137 k_jacobi, then r = b - A x
                b = S.rhs[t];
                if (mean != 0.0f) {
                    b = __fsub_rn(b, mean);
                    S.rhs[t] = b;
                }
                float s = 0.0f;
                if (i > 0) s = __fadd_rn(s, S.ax[uidx_(n, i, j, k)]);
                if (i < n - 1) s = __fadd_rn(s, S.ax[uidx_(n, i + 1, j, k)]);
                if (j > 0) s = __fadd_rn(s, S.ay[vidx_(n, i, j, k)]);
                if (j < n - 1) s = __fadd_rn(s, S.ay[vidx_(n, i, j + 1, k)]);
                if (k > 0) s = __fadd_rn(s, S.az[widx_(n, i, j, k)]);
                if (k < n - 1) s = __fadd_rn(s, S.az[widx_(n, i, j, k + 1)]);
                d = __fdiv_rn(hh, maxf_(s, 1.0e-12f));
                S.pdiag[t] = d;
                r = __fsub_rn(b, __fdiv_rn(lap_acc(S, X, xc, t, i, j, k), hh));
            }
            const float z = __fmul_rn(d, r);
            S.cg_r[t] = r;
            S.cg_z[t] = z;
            part[0] += (double)b * (double)b;
            part[1] += (double)r * (double)r;
            part[2] += (double)r * (double)z;
        }
        put_partials<3>(bufB, c, part, red);
    }
    if (!grid_barrier(bar, epoch, ws.err)) goto finish;

    // ------------------------------------------------------------------------------------------ iterations
    for (int kit = 1;; ++kit) {
        // scene scalars from the previous phase B (or the prologue): convergence test, beta
        for (int s = s_lo; s <= s_hi; ++s) {
            LocalScene& L = loc[s - s_lo];
            const hf_scene& S = scenes[s];
            const int b = ws.chunk_begin[s], e = ws.chunk_begin[s + 1];
            const bool owner = b >= c0 && b < c1;
            if (kit == 1) {
                double tot[3];
                const int comp[3] = {0, 1, 2};
                scene_sums<3>(bufB, b, e, comp, tot, red);
                if (threadIdx.x == 0) {
                    const int n = S.n;
                    const double tol = HEAT ? S.heat_tol : S.cg_tol;
                    double atol = tol * sqrt(tot[0]);
                    if (atol < tol) atol = tol;
                    if (atol < 1.0e-18) atol = 1.0e-18;
                    int maxit = HEAT ? S.heat_maxiter : S.cg_max_iter;
                    if (maxit <= 0) maxit = n * n * n;
                    L.maxit = maxit + (maxit & 1);   // iterations run in pairs
                    L.bb = tot[0];
                    L.rr = tot[1];
                    L.rz = tot[2];
                    L.atol_sq = atol * atol;
                    L.iters = 0;
                    L.beta = 0.0f;
                    L.status = isfinite(tot[1]) ? 0 : HF_SCENE_NONFINITE;
                    L.live = (b < e) && tot[1] > L.atol_sq && isfinite(tot[1]) && L.maxit > 0;
                    if (owner && L.live) atomicAdd(live_count, 1u);
                }
            } else {
                if (!loc[s - s_lo].live) continue;   // uniform: read by all threads after the last __syncthreads
                double tot[2];
                const int comp[2] = {1, 2};
                scene_sums<2>(bufB, b, e, comp, tot, red);
                if (threadIdx.x == 0) {
                    const double rr = tot[0], rz = tot[1];
                    L.iters = kit - 1;
                    const bool above = rr > L.atol_sq;
                    L.beta = above ? __double2float_rn(rz / L.rz) : 0.0f;
                    L.rz = rz;
                    L.rr = rr;
                    if (!isfinite(rr)) L.status |= HF_SCENE_NONFINITE;
                    const bool live = above && isfinite(rr) && L.iters < L.maxit;
                    if (!live) {
                        if (above && isfinite(rr)) L.status |= HEAT ? HF_SCENE_HEAT_MAXITER : HF_SCENE_PRESSURE_MAXITER;
                        L.live = 0;
                        if (owner) atomicSub(live_count, 1u);
                    }
                }
            }
            __syncthreads();
            if (owner && threadIdx.x == 0 && !L.live) {
                CgCtl& W = ws.ctl[s];
                W.bb = L.bb;
                W.rr = L.rr;
                W.atol_sq = L.atol_sq;
                W.iters = L.iters;
                W.status = L.status;
                if (!HEAT) W.mean = L.mean;
            }
            __syncthreads();
        }
        // phase A: p_k at the stencil points, Ap = A p_k, p.Ap
        for (int c = c0; c < c1; ++c) {
            const WorkItem wi = work[c];
            const LocalScene& L = loc[wi.scene - s_lo];
            if (!L.live) continue;
            const hf_scene& S = scenes[wi.scene];
            const int n = S.n, N = n * n * n;
            const float h = (float)S.h, hh = __fmul_rn(h, h), c_dt = __fdiv_rn(dt, hh);
            const Dir P{S.cg_z, S.cg_p[(kit - 1) & 1], L.beta, kit == 1};
            float pc[kCellsPerThread], ap[kCellsPerThread];
            // all loads of the thread's cells first, stores after: keeps every cell's loads in flight together
#pragma unroll
            for (int m = 0; m < kCellsPerThread; ++m) {
                const int t = wi.first + threadIdx.x + m * kThreads;
                pc[m] = 0.0f;
                ap[m] = 0.0f;
                if (t < N) {
                    int i, j, k;
                    cell_ijk(t, n, i, j, k);
                    pc[m] = P(t);
                    if (HEAT) {
                        ap[m] = (__ldg(S.cell_flags + t) & 1) ? pc[m]
                                                              : __fadd_rn(pc[m], __fmul_rn(c_dt, heat_nt(S, P, pc[m], t, i, j, k)));
                    } else {
                        ap[m] = __fdiv_rn(lap_acc(S, P, pc[m], t, i, j, k), hh);
                    }
                }
            }
            float* pnew = S.cg_p[kit & 1];
            double part[1] = {0.0};
#pragma unroll
            for (int m = 0; m < kCellsPerThread; ++m) {
                const int t = wi.first + threadIdx.x + m * kThreads;
                if (t < N) {
                    pnew[t] = pc[m];
                    S.cg_Ap[t] = ap[m];
                    part[0] += (double)pc[m] * (double)ap[m];
                }
            }
            put_partials<1>(bufA, c, part, red);
        }
        if (!grid_barrier(bar, epoch, ws.err)) goto finish;
        if (*(volatile unsigned*)live_count == 0u) break;
        // alpha = r.z / p.Ap of every live scene
        for (int s = s_lo; s <= s_hi; ++s) {
            LocalScene& L = loc[s - s_lo];
            if (!L.live) continue;
            double tot[1];
            const int comp[1] = {0};
            scene_sums<1>(bufA, ws.chunk_begin[s], ws.chunk_begin[s + 1], comp, tot, red);
            if (threadIdx.x == 0) {
                L.pAp = tot[0];
                L.alpha = __double2float_rn(L.rz / tot[0]);
            }
            __syncthreads();
        }
        // phase B: x += alpha p, r -= alpha Ap, z = D r, r.r and r.z
        for (int c = c0; c < c1; ++c) {
            const WorkItem wi = work[c];
            const LocalScene& L = loc[wi.scene - s_lo];
            if (!L.live) continue;
            const hf_scene& S = scenes[wi.scene];
            const int n = S.n, N = n * n * n, par = s_par[wi.scene];
            float* x = HEAT ? S.T[par ^ 1] : S.p;
            const float* D = HEAT ? S.hdiag : S.pdiag;
            const float* pk = S.cg_p[kit & 1];
            const float alpha = L.alpha;
            float xv[kCellsPerThread], rv[kCellsPerThread], zv[kCellsPerThread];
#pragma unroll
            for (int m = 0; m < kCellsPerThread; ++m) {
                const int t = wi.first + threadIdx.x + m * kThreads;
                if (t < N) {
                    xv[m] = __fadd_rn(x[t], __fmul_rn(alpha, pk[t]));
                    rv[m] = __fsub_rn(S.cg_r[t], __fmul_rn(alpha, S.cg_Ap[t]));
                    zv[m] = __fmul_rn(D[t], rv[m]);
                }
            }
            double part[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int m = 0; m < kCellsPerThread; ++m) {
                const int t = wi.first + threadIdx.x + m * kThreads;
                if (t < N) {
                    x[t] = xv[m];
                    S.cg_r[t] = rv[m];
                    S.cg_z[t] = zv[m];
                    part[1] += (double)rv[m] * (double)rv[m];
                    part[2] += (double)rv[m] * (double)zv[m];
                }
            }
            put_partials<3>(bufB, c, part, red);
        }
        if (!grid_barrier(bar, epoch, ws.err)) goto finish;
    }

    // -------------------------------------------------------------------- pressure epilogue: projection
    if (!HEAT) {
        // grid.py:140-153 k_project x3 with dt/rho formed in double (grid.py:251)
        for (int c = c0; c < c1; ++c) {
            const WorkItem wi = work[c];
            const hf_scene& S = scenes[wi.scene];
            const int n = S.n, N = n * n * n, nn = n * n, par = s_par[wi.scene];
            const float h = (float)S.h, dtr = (float)(dt_d / S.rho);
            float *u = S.u[par ^ 1], *v = S.v[par ^ 1], *w = S.w[par ^ 1];
            const float* p = S.p;
            for (int m = 0; m < kCellsPerThread; ++m) {
                const int t = wi.first + threadIdx.x + m * kThreads;
                if (t >= N) break;
                int i, j, k;
                cell_ijk(t, n, i, j, k);
                const float pc = p[t];
                int f = uidx_(n, i, j, k);
                u[f] = i == 0 ? 0.0f : __fsub_rn(u[f], __fdiv_rn(__fmul_rn(dtr, __fsub_rn(pc, p[t - nn])), h));
                f = vidx_(n, i, j, k);
                v[f] = j == 0 ? 0.0f : __fsub_rn(v[f], __fdiv_rn(__fmul_rn(dtr, __fsub_rn(pc, p[t - n])), h));
                f = widx_(n, i, j, k);
                w[f] = k == 0 ? 0.0f : __fsub_rn(w[f], __fdiv_rn(__fmul_rn(dtr, __fsub_rn(pc, p[t - 1])), h));
                if (i == n - 1) u[uidx_(n, n, j, k)] = 0.0f;
                if (j == n - 1) v[vidx_(n, i, n, k)] = 0.0f;
                if (k == n - 1) w[widx_(n, i, j, n)] = 0.0f;
            }
        }
    }

finish:
    // statistics (and, after the pressure solve, the end of the substep).  Owners wrote their scene records before
    // the last barrier; every block read the parities before its first barrier, so block 0 may flip them now.
    if (blockIdx.x == 0) {
        const bool timed_out = *(volatile int*)ws.err != 0;
        for (int s = threadIdx.x; s < num_scenes; s += kThreads) {
            const hf_scene& S = scenes[s];
            if (!(S.flags & HF_FLAG_ACTIVE)) continue;
            const CgCtl& C = ws.ctl[s];
            hf_scene_state* st = S.state;
            if (HEAT) {
                st->status = C.status | (timed_out ? HF_SCENE_BARRIER_TIMEOUT : 0);
                st->heat_iters = C.iters;
                st->heat_rr = C.rr;
                st->heat_atol = sqrt(C.atol_sq);
                st->heat_bb = C.bb;
                st->total_heat_iters += C.iters;
            } else {
                st->status |= C.status | (timed_out ? HF_SCENE_BARRIER_TIMEOUT : 0);
                st->pressure_iters = C.iters;
                st->pressure_rr = C.rr;
                st->pressure_atol = sqrt(C.atol_sq);
                st->pressure_bb = C.bb;
                st->rhs_mean = C.mean;
                st->total_pressure_iters += C.iters;
                if (!timed_out) {
                    st->parity = s_par[s] ^ 1;
                    st->substeps += 1;
                }
            }
        }
    }
}

// ================================================================================ register-resident variant
// Single-scene plans whose chunks fit one block per SM keep the whole CG state of their cells in registers: every
// thread owns the same cells for the entire solve (x, r, z, p, D and Ap never leave the SM); per iteration only the
// search direction p (phase A) and z (phase B) are published to global memory, because neighbouring blocks read them
// at their stencil points.  The chunk -> (group, thread) mapping and the reduction tree are those of k_pcg (256
// virtual threads x 4 cells per chunk, warp butterfly, 8 warps in order), so both kernels produce the same bits.
//
// Block = `groups` x 256 threads; group g owns chunks c0 + g + groups*q (q < MAXC) of the block's contiguous range.
template <int K>
__device__ __forceinline__ void group_sum(double (&v)[K], double* red) {
    // red: K * (blockDim.x / 32) doubles; every 256-thread group reduces its own 8 warps in index order
#pragma unroll
    for (int c = 0; c < K; ++c) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_xor_sync(0xffffffffu, v[c], o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int g0 = (warp >> 3) << 3;   // first warp of this group
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int c = 0; c < K; ++c) red[c * nw + warp] = v[c];
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < K; ++c) {
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < 8; ++q) s += red[c * nw + g0 + q];
        v[c] = s;
    }
}

// scene_sums for blocks of any size: the first 256 threads form the same tree as scene_sums in a 256-thread block.
template <int K>
__device__ __forceinline__ void scene_sums_g(const double* __restrict__ buf, int b, int e, const int (&comp)[K],
                                             double (&tot)[K], double* red) {
#pragma unroll
    for (int q = 0; q < K; ++q) tot[q] = 0.0;
    if (threadIdx.x < kThreads) {
        for (int c = b + threadIdx.x; c < e; c += kThreads) {
#pragma unroll
            for (int q = 0; q < K; ++q) tot[q] += buf[3 * c + comp[q]];
        }
    }
#pragma unroll
    for (int c = 0; c < K; ++c) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) tot[c] += __shfl_xor_sync(0xffffffffu, tot[c], o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0 && warp < kThreads / 32) {
#pragma unroll
        for (int c = 0; c < K; ++c) red[c * (kThreads / 32) + warp] = tot[c];
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < K; ++c) {
        double sum = 0.0;
#pragma unroll
        for (int q = 0; q < kThreads / 32; ++q) sum += red[c * (kThreads / 32) + q];
        tot[c] = sum;
    }
}

template <bool HEAT, int MAXC>
__global__ void __launch_bounds__(MAXC == 1 ? 1024 : (MAXC == 2 ? 768 : 512), 1) k_pcg_res(const hf_scene* __restrict__ scenes, const WorkItem* __restrict__ work,
                                                    int num_chunks, int num_scenes, double dt_d, Workspace ws) {
    constexpr int CPT = kCellsPerThread * MAXC;   // cells per thread
    __shared__ double red[3 * 32];
    __shared__ LocalScene Ls;
    const int groups = blockDim.x >> 8, g = threadIdx.x >> 8, lt = threadIdx.x & 255;
    const int c0 = (int)(((long long)num_chunks * blockIdx.x) / gridDim.x);
    const int c1 = (int)(((long long)num_chunks * (blockIdx.x + 1)) / gridDim.x);
    const int sidx = work[c0].scene;                       // one scene per plan on this path
    const hf_scene& S = scenes[sidx];
    const int n = S.n, N = n * n * n, nn = n * n;
    const int par = S.state->parity;
    unsigned* bar = ws.bar + (HEAT ? 0 : 1);
    unsigned epoch = 0;
    const float dt = (float)dt_d;
    const float h = (float)S.h, hh = __fmul_rn(h, h), c_dt = __fdiv_rn(dt, hh);
    double* bufA = ws.partials;
    double* bufB = ws.partials + 3 * (size_t)num_chunks;
    const int cb = ws.chunk_begin[sidx], ce = ws.chunk_begin[sidx + 1];
    float* xg = HEAT ? S.T[par ^ 1] : S.p;
    float* zg = S.cg_z;

    // cells of this thread: chunk q, sub-cell m -> slot q*4+m (chunks of a one-scene plan are consecutive)
    float x[CPT], r[CPT], z[CPT], p[CPT], D[CPT], Ap[CPT];
    const int cell0 = (c0 + g - cb) * kChunk + lt;
    const int cstep = groups * kChunk;
    const int clim = min(N, (c1 - cb) * kChunk);
#define TCELL(s_) (cell0 + ((s_) / kCellsPerThread) * cstep + ((s_) % kCellsPerThread) * kThreads)
#define TVALID(t_) ((t_) < clim)
    // ------------------------------------------------------------------ prologue (as k_pcg, values kept in regs)
    float mean = 0.0f;
    if (!HEAT) {
        double mm[1];
        const int comp[1] = {0};
        scene_sums_g<1>(bufA, cb, ce, comp, mm, red);   
        mean = __double2float_rn(mm[0] / ((double)n * n * n));
    }
    {
        const Vec X{xg};
#pragma unroll
        for (int s = 0; s < CPT; ++s) {
            x[s] = r[s] = z[s] = p[s] = D[s] = Ap[s] = 0.0f;
            const int t = TCELL(s);
            if (!TVALID(t)) continue;
            int i, j, k;
            cell_ijk(t, n, i, j, k);
            float b, d, rr;
            const float xc = xg[t];
            if (HEAT) {
                b = S.hrhs[t];
                if (S.cell_flags[t] & 1) {
                    d = 1.0f;
                    rr = __fsub_rn(b, xc);
                } else {
                    d = __fdiv_rn(1.0f, __fadd_rn(1.0f, __fmul_rn(c_dt, heat_diag_sum(S, i, j, k))));
                    rr = __fsub_rn(b, __fadd_rn(xc, __fmul_rn(c_dt, heat_nt(S, X, xc, t, i, j, k))));
                }
            } else {
                b = S.rhs[t];
                if (mean != 0.0f) {
                    b = __fsub_rn(b, mean);
                    S.rhs[t] = b;
                }
                float sa = 0.0f;
                if (i > 0) sa = __fadd_rn(sa, S.ax[uidx_(n, i, j, k)]);
                if (i < n - 1) sa = __fadd_rn(sa, S.ax[uidx_(n, i + 1, j, k)]);
                if (j > 0) sa = __fadd_rn(sa, S.ay[vidx_(n, i, j, k)]);
                if (j < n - 1) sa = __fadd_rn(sa, S.ay[vidx_(n, i, j + 1, k)]);
                if (k > 0) sa = __fadd_rn(sa, S.az[widx_(n, i, j, k)]);
                if (k < n - 1) sa = __fadd_rn(sa, S.az[widx_(n, i, j, k + 1)]);
                d = __fdiv_rn(hh, maxf_(sa, 1.0e-12f));
                rr = __fsub_rn(b, __fdiv_rn(lap_acc(S, X, xc, t, i, j, k), hh));
            }
            x[s] = xc;
            D[s] = d;
            r[s] = rr;
            z[s] = __fmul_rn(d, rr);
            Ap[s] = b;   // holds b until the partial sums below
        }
    }
#pragma unroll
    for (int q = 0; q < MAXC; ++q) {
        double part[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int m = 0; m < kCellsPerThread; ++m) {
            const int s = q * kCellsPerThread + m, t = TCELL(s);
            if (!TVALID(t)) continue;
            zg[t] = z[s];
            part[0] += (double)Ap[s] * (double)Ap[s];
            part[1] += (double)r[s] * (double)r[s];
            part[2] += (double)r[s] * (double)z[s];
        }
        group_sum<3>(part, red);
        const int c = c0 + g + groups * q;
        if (lt == 0 && c < c1) {
            bufB[3 * c] = part[0];
            bufB[3 * c + 1] = part[1];
            bufB[3 * c + 2] = part[2];
        }
    }
    if (!grid_barrier(bar, epoch, ws.err)) goto finish;
    {
        double tot[3];
        const int comp[3] = {0, 1, 2};
        scene_sums_g<3>(bufB, cb, ce, comp, tot, red);
        if (threadIdx.x == 0) {
            const double tol = HEAT ? S.heat_tol : S.cg_tol;
            double atol = tol * sqrt(tot[0]);
            if (atol < tol) atol = tol;
            if (atol < 1.0e-18) atol = 1.0e-18;
            int maxit = HEAT ? S.heat_maxiter : S.cg_max_iter;
            if (maxit <= 0) maxit = N;
            Ls.maxit = maxit + (maxit & 1);
            Ls.bb = tot[0];
            Ls.rr = tot[1];
            Ls.rz = tot[2];
            Ls.atol_sq = atol * atol;
            Ls.iters = 0;
            Ls.beta = 0.0f;
            Ls.mean = (double)mean;
            Ls.status = isfinite(tot[1]) ? 0 : HF_SCENE_NONFINITE;
            Ls.live = tot[1] > Ls.atol_sq && isfinite(tot[1]) && Ls.maxit > 0;
        }
        __syncthreads();
    }
    // ------------------------------------------------------------------------------------------ iterations
    for (int kit = 1; Ls.live; ++kit) {
        // phase A: p_k (own cells from registers, neighbours from z and p_{k-1} in global memory), Ap, p.Ap
        const float beta = Ls.beta;
        const bool first = kit == 1;
        const float* pold = S.cg_p[(kit - 1) & 1];
        float* pnew = S.cg_p[kit & 1];
        const Dir P{zg, pold, beta, first};
#pragma unroll
        for (int s = 0; s < CPT; ++s) {
            const int t = TCELL(s);
            if (!TVALID(t)) continue;
            const float pc = first ? z[s] : __fadd_rn(z[s], __fmul_rn(beta, p[s]));
            int i, j, k;
            cell_ijk(t, n, i, j, k);
            if (HEAT) {
                Ap[s] = (__ldg(S.cell_flags + t) & 1) ? pc : __fadd_rn(pc, __fmul_rn(c_dt, heat_nt(S, P, pc, t, i, j, k)));
            } else {
                Ap[s] = __fdiv_rn(lap_acc(S, P, pc, t, i, j, k), hh);
            }
            p[s] = pc;
        }
#pragma unroll
        for (int q = 0; q < MAXC; ++q) {
            double part[1] = {0.0};
#pragma unroll
            for (int m = 0; m < kCellsPerThread; ++m) {
                const int s = q * kCellsPerThread + m, t = TCELL(s);
                if (!TVALID(t)) continue;
                pnew[t] = p[s];
                part[0] += (double)p[s] * (double)Ap[s];
            }
            group_sum<1>(part, red);
            const int c = c0 + g + groups * q;
            if (lt == 0 && c < c1) bufA[3 * c] = part[0];
        }
        if (!grid_barrier(bar, epoch, ws.err)) goto finish;
        {
            double tot[1];
            const int comp[1] = {0};
            scene_sums_g<1>(bufA, cb, ce, comp, tot, red);
            if (threadIdx.x == 0) {
                Ls.pAp = tot[0];
                Ls.alpha = __double2float_rn(Ls.rz / tot[0]);
            }
            __syncthreads();
        }
        // phase B: x += alpha p, r -= alpha Ap, z = D r (registers), publish z, r.r and r.z
        const float alpha = Ls.alpha;
#pragma unroll
        for (int q = 0; q < MAXC; ++q) {
            double part[2] = {0.0, 0.0};
#pragma unroll
            for (int m = 0; m < kCellsPerThread; ++m) {
                const int s = q * kCellsPerThread + m, t = TCELL(s);
                if (!TVALID(t)) continue;
                x[s] = __fadd_rn(x[s], __fmul_rn(alpha, p[s]));
                r[s] = __fsub_rn(r[s], __fmul_rn(alpha, Ap[s]));
                z[s] = __fmul_rn(D[s], r[s]);
                zg[t] = z[s];
                part[0] += (double)r[s] * (double)r[s];
                part[1] += (double)r[s] * (double)z[s];
            }
            group_sum<2>(part, red);
            const int c = c0 + g + groups * q;
            if (lt == 0 && c < c1) {
                bufB[3 * c + 1] = part[0];
                bufB[3 * c + 2] = part[1];
            }
        }
        if (!grid_barrier(bar, epoch, ws.err)) goto finish;
        {
            double tot[2];
            const int comp[2] = {1, 2};
            scene_sums_g<2>(bufB, cb, ce, comp, tot, red);
            if (threadIdx.x == 0) {
                const double rr = tot[0], rz = tot[1];
                Ls.iters = kit;
                const bool above = rr > Ls.atol_sq;
                Ls.beta = above ? __double2float_rn(rz / Ls.rz) : 0.0f;
                Ls.rz = rz;
                Ls.rr = rr;
                if (!isfinite(rr)) Ls.status |= HF_SCENE_NONFINITE;
                const bool live = above && isfinite(rr) && kit < Ls.maxit;
                if (!live && above && isfinite(rr)) Ls.status |= HEAT ? HF_SCENE_HEAT_MAXITER : HF_SCENE_PRESSURE_MAXITER;
                Ls.live = live;
            }
            __syncthreads();
        }
    }
    // ------------------------------------------------------------------ write the solution back
#pragma unroll
    for (int s = 0; s < CPT; ++s)
        if (TVALID(TCELL(s))) xg[TCELL(s)] = x[s];
    if (!HEAT) {
        // grid.py:140-153: the projection reads p at neighbour cells owned by other blocks
        if (!grid_barrier(bar, epoch, ws.err)) goto finish;
        const float dtr = (float)(dt_d / S.rho);
        float *u = S.u[par ^ 1], *v = S.v[par ^ 1], *w = S.w[par ^ 1];
        const float* pp = S.p;
#pragma unroll
        for (int s = 0; s < CPT; ++s) {
            const int t = TCELL(s);
            if (!TVALID(t)) continue;
            int i, j, k;
            cell_ijk(t, n, i, j, k);
            const float pc = x[s];
            int f = uidx_(n, i, j, k);
            u[f] = i == 0 ? 0.0f : __fsub_rn(u[f], __fdiv_rn(__fmul_rn(dtr, __fsub_rn(pc, pp[t - nn])), h));
            f = vidx_(n, i, j, k);
            v[f] = j == 0 ? 0.0f : __fsub_rn(v[f], __fdiv_rn(__fmul_rn(dtr, __fsub_rn(pc, pp[t - n])), h));
            f = widx_(n, i, j, k);
            w[f] = k == 0 ? 0.0f : __fsub_rn(w[f], __fdiv_rn(__fmul_rn(dtr, __fsub_rn(pc, pp[t - 1])), h));
            if (i == n - 1) u[uidx_(n, n, j, k)] = 0.0f;
            if (j == n - 1) v[vidx_(n, i, n, k)] = 0.0f;
            if (k == n - 1) w[widx_(n, i, j, n)] = 0.0f;
        }
    }
finish:
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const bool timed_out = *(volatile int*)ws.err != 0;
        hf_scene_state* st = S.state;
        if (HEAT) {
            st->status = Ls.status | (timed_out ? HF_SCENE_BARRIER_TIMEOUT : 0);
            st->heat_iters = Ls.iters;
            st->heat_rr = Ls.rr;
            st->heat_atol = sqrt(Ls.atol_sq);
            st->heat_bb = Ls.bb;
            st->total_heat_iters += Ls.iters;
        } else {
            st->status |= Ls.status | (timed_out ? HF_SCENE_BARRIER_TIMEOUT : 0);
            st->pressure_iters = Ls.iters;
            st->pressure_rr = Ls.rr;
            st->pressure_atol = sqrt(Ls.atol_sq);
            st->pressure_bb = Ls.bb;
            st->rhs_mean = Ls.mean;
            st->total_pressure_iters += Ls.iters;
            if (!timed_out) {
                st->parity = par ^ 1;
                st->substeps += 1;
            }
        }
    }
}

#undef TCELL
#undef TVALID

const void* pcg_resident_kernel(bool heat, int maxc) {
    if (heat) {
        if (maxc == 1) return (const void*)k_pcg_res<true, 1>;
        if (maxc == 2) return (const void*)k_pcg_res<true, 2>;
        return (const void*)k_pcg_res<true, 3>;
    }
    if (maxc == 1) return (const void*)k_pcg_res<false, 1>;
    if (maxc == 2) return (const void*)k_pcg_res<false, 2>;
    return (const void*)k_pcg_res<false, 3>;
}

const void* pcg_kernel(bool heat) { return heat ? (const void*)k_pcg<true> : (const void*)k_pcg<false>; }

}  // namespace hf
