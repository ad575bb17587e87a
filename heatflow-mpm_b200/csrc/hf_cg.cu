// hf_cg.cu -- persistent, cooperative Jacobi-preconditioned CG for the heat and pressure systems of a batch of scenes.
//
// One launch performs a whole solve (heat.py:198-210 or grid.py:235-251) with the convergence test on the device, so
// no iteration waits for the host.  The grid is co-resident (cooperative launch); phases are separated by a software
// grid barrier whose wait is bounded in time (a timeout sets a flag and every block leaves the solve).
//
// Semantics follow warp.optim.linear.cg with M = diag(D) (warp-lang, a dependency of the reference; restated from its
// published algorithm):
//     r = b - A x,  z = D r,  p = z,  atol = max(tol ||b||, tol, 1e-18)
//     repeat: Ap = A p; alpha = rz / pAp; x += alpha p; r -= alpha Ap; z = D r; beta = rz'/rz; p = z + beta p
//     until r.r <= atol^2 (tested every iteration, which is where the reference's frozen iterations leave x) or maxiter.
// Inner products, alpha and beta are fp64; the vectors stay binary32 and alpha/beta are applied after rounding.
//
// Work items are 4 x 8 x 32-cell tiles (i, j, k).  Thread lt of a tile owns cells (i0 + m, j0 + lt/32, k0 + lt%32),
// m = 0..3, so a warp covers one 128-byte k-row.  Each tile yields one fp64 partial per inner product in a fixed tree
// (4 cells in order, warp butterfly, 8 warps in order); a scene's inner product sums its tile partials in tile order
// (again a fixed tree).  Results therefore depend only on the scene -- not on the batch, the grid size or the variant.
//
// Two grid barriers per iteration: the search direction p_k = z + beta p_{k-1} is not a separate phase -- every block
// recomputes it at the stencil points it reads from z and the previous p (double-buffered), so it costs no barrier.
//
// Variants:
//   k_pcg       streaming: vectors in global memory, any number of scenes (batched and served plans).  The scenes come
//               in L2-sized groups solved by the lanes of the grid; for the pressure system with every scene at
//               n % 4 == 0 each tile's stencil boxes and CG vectors are staged by TMA from per-scene descriptors,
//               double-buffered per block.  Optional outer defect correction (fp64 true residual, restart).
//   k_pcg_res   register-resident, one scene: every thread keeps x, r, z, p, D and Ap of its cells in registers for
//               the whole solve; only p and z are published (neighbouring blocks read them).
//   k_pcg_tma   register-resident pressure solve of one scene with n % 4 == 0: the stencil inputs of each tile -- z
//               and the previous p with a one-cell halo, and the face fractions -- are staged into shared memory by
//               TMA (cp.async.bulk.tensor) instead of gathered; x, r and D stay in registers.
#include <cuda.h>

#include "hf_device.cuh"
#include "hf_kernels.cuh"

namespace hf {

constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;   // 2 s
// Limit of every bounded wait of the CG kernels (grid and lane barriers, TMA copies), and the block that does not
// arrive at the first grid barrier of each persistent CG launch (-1: none).  The defaults are what every solve uses;
// hf_set_wait_limit changes both, so that a test can make a barrier's wait run out on purpose and check that the
// kernel reports HF_SCENE_BARRIER_TIMEOUT and returns with the context usable.
__constant__ unsigned long long c_wait_limit_ns = kBarrierTimeoutNs;
__constant__ int c_absent_block = -1;
// Components one group_sum / scene_sums call reduces at most: 3 inner products per tile x 3 tiles of a 256-thread
// group (the resident variants' set-up).  Every CG kernel's `red` holds kRedComps x 32 doubles (one per warp).
constexpr int kRedComps = 9;
constexpr int kMaxCorrections = 2;   // restarts of one solve by the outer defect correction

__device__ __forceinline__ int uidx_(int n, int i, int j, int k) { return (i * n + j) * n + k; }
__device__ __forceinline__ int vidx_(int n, int i, int j, int k) { return (i * (n + 1) + j) * n + k; }
__device__ __forceinline__ int widx_(int n, int i, int j, int k) { return (i * n + j) * (n + 1) + k; }

// Barrier of nblocks blocks (the grid, or one lane of it) with a bounded wait.  Thread 0 publishes the block's writes with a release reduction (cumulative over
// the writes the block's threads made before __syncthreads) and polls with acquire loads.  Returns false (in every
// thread) once any block has timed out.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned& epoch, int* err, unsigned nblocks) {
    ++epoch;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned target = epoch * nblocks;
        if (!(epoch == 1 && (int)blockIdx.x == c_absent_block))
            asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(bar) : "memory");
        const unsigned long long t0 = global_timer_ns(), limit = c_wait_limit_ns;
        unsigned spins = 0;
        while (ld_acquire_u32(bar) < target) {
            if (*(volatile int*)err) break;
            if ((++spins & 255u) == 0 && global_timer_ns() - t0 > limit) {
                atomicExch(err, 1);
                break;
            }
        }
    }
    __syncthreads();
    return *(volatile int*)err == 0;
}

// Sum of a scene's partials (item c, component comp[q] at buf[comp[q] * cs + c]: component-major, so that a warp's
// loads of one component are contiguous) in a fixed tree: the first 256 threads stride over the items in order, warp
// butterfly, then 8 warps in order.  Every block computing it obtains the same bits.  cs is the plan's tile count for
// the tile partials (three components, see part_idx) and 0 for the per-chunk rhs sums (one component).
template <int K, int U = 4>
__device__ __forceinline__ void scene_sums(const double* __restrict__ buf, int b, int e, const int (&comp)[K],
                                           double (&tot)[K], double* red, int cs) {
    static_assert(K <= kRedComps, "red holds kRedComps components");
#pragma unroll
    for (int q = 0; q < K; ++q) tot[q] = 0.0;
    if (threadIdx.x < kThreads) {
        // a thread's partials c = b + t, b + t + 256, ... are added in that order; U at a time are loaded (an absent
        // one as +0.0, which leaves a sum that started at +0.0 unchanged) before they are added, so their L2 round
        // trips overlap instead of each waiting for the previous addition
        for (int c = b + threadIdx.x; c < e; c += U * kThreads) {
            double v[U][K];
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int q = 0; q < K; ++q) v[u][q] = c + u * kThreads < e ? buf[comp[q] * cs + c + u * kThreads] : 0.0;
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int q = 0; q < K; ++q) tot[q] += v[u][q];
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
        for (int c = 0; c < K; ++c) red[c * 32 + warp] = tot[c];
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < K; ++c) {
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < kThreads / 32; ++q) s += red[c * 32 + q];
        tot[c] = s;
    }
}

// scene_sums for every live scene q < ns of a group (scene scene_lo + q: items tile_begin[s] .. tile_begin[s + 1]), with
// the same tree per scene, in passes of kRedComps * 32 / (8 K) scenes that share one pair of block barriers instead of
// a pair per scene; fn(q, tot) then runs once per live scene, in one thread, with the scene's K sums.  live(q) must
// not change before fn runs for q.  256-thread blocks.
template <int K, class Live, class Fn>
__device__ __forceinline__ void group_sums(const double* __restrict__ buf, const int* __restrict__ tile_begin,
                                           int scene_lo, int ns, const int (&comp)[K], int cs, double* red, Live live,
                                           Fn fn) {
    constexpr int CH = kRedComps * 32 / (8 * K);
    const int lt = threadIdx.x, lane = lt & 31, warp = lt >> 5;
    for (int q0 = 0; q0 < ns; q0 += CH) {
        const int qn = ns - q0 < CH ? ns - q0 : CH;
        for (int qq = 0; qq < qn; ++qq) {
            if (!live(q0 + qq)) continue;
            const int b = tile_begin[scene_lo + q0 + qq], e = tile_begin[scene_lo + q0 + qq + 1];
            double acc[K];
#pragma unroll
            for (int k = 0; k < K; ++k) acc[k] = 0.0;
            for (int c = b + lt; c < e; c += 4 * kThreads) {
                double v[4][K];
#pragma unroll
                for (int u = 0; u < 4; ++u)
#pragma unroll
                    for (int k = 0; k < K; ++k) v[u][k] = c + u * kThreads < e ? buf[comp[k] * cs + c + u * kThreads] : 0.0;
#pragma unroll
                for (int u = 0; u < 4; ++u)
#pragma unroll
                    for (int k = 0; k < K; ++k) acc[k] += v[u][k];
            }
#pragma unroll
            for (int k = 0; k < K; ++k) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
            }
            if (lane == 0) {
#pragma unroll
                for (int k = 0; k < K; ++k) red[(qq * K + k) * 8 + warp] = acc[k];
            }
        }
        __syncthreads();
        if (lt < qn && live(q0 + lt)) {
            double tot[K];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                double t = 0.0;
#pragma unroll
                for (int w = 0; w < kThreads / 32; ++w) t += red[(lt * K + k) * 8 + w];
                tot[k] = t;
            }
            fn(q0 + lt, tot);
        }
        __syncthreads();
    }
}

// Per-256-thread-group sum (each group reduces its own 8 warps in index order): the tile partial tree.
template <int K>
__device__ __forceinline__ void group_sum(double (&v)[K], double* red) {
    static_assert(K <= kRedComps, "red holds kRedComps components");
#pragma unroll
    for (int c = 0; c < K; ++c) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_xor_sync(0xffffffffu, v[c], o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g0 = (warp >> 3) << 3;
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int c = 0; c < K; ++c) red[c * 32 + warp] = v[c];
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < K; ++c) {
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < 8; ++q) s += red[c * 32 + g0 + q];
        v[c] = s;
    }
}

// group_sum in two steps, so that a thread holds the partials of one tile at a time: stash_warp reduces K values over the
// warp (the same butterfly) and lane 0 parks them in red[(c0 + c) * 32 + warp]; after every tile's stash,
// publish_group (thread lt == 0 of each 256-thread group) adds the group's 8 warps in order -- group_sum's tree, the
// same bits -- and writes the tile partials to buf[c * tiles + tile] (3 components, component-major).  red must not be read by
// another phase in between (the caller's barriers see to that).
template <int K>
__device__ __forceinline__ void stash_warp(double (&v)[K], double* red, int c0) {
#pragma unroll
    for (int c = 0; c < K; ++c) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_xor_sync(0xffffffffu, v[c], o);
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int c = 0; c < K; ++c) red[(c0 + c) * 32 + (threadIdx.x >> 5)] = v[c];
    }
}

template <int MAXC>
__device__ __forceinline__ void publish_group(const double* red, double* __restrict__ buf, int first_tile, int groups,
                                              int c_end, int tiles) {
    __syncthreads();
    if ((threadIdx.x & 255) == 0) {
        const int g0 = (threadIdx.x >> 5);   // first warp of this group
#pragma unroll
        for (int q = 0; q < MAXC; ++q) {
            const int c = first_tile + groups * q;
            if (c >= c_end) continue;
#pragma unroll
            for (int comp = 0; comp < 3; ++comp) {
                double s = 0.0;
#pragma unroll
                for (int w = 0; w < 8; ++w) s += red[(3 * q + comp) * 32 + g0 + w];
                buf[comp * tiles + c] = s;
            }
        }
    }
}

// One partial per 256-thread group (the single-reduction CG's five components), stored component-major so that a
// warp's loads of one component are contiguous: after stash_warp<K>(v, red, 0) in every warp, thread lt == 0 of each
// group adds its 8 warps in order and writes buf[comp * units + unit].
template <int K>
__device__ __forceinline__ void publish_unit(const double* red, double* __restrict__ buf, int unit, int units) {
    __syncthreads();
    if ((threadIdx.x & 255) == 0) {
        const int g0 = (threadIdx.x >> 5);
#pragma unroll
        for (int comp = 0; comp < K; ++comp) {
            double s = 0.0;
#pragma unroll
            for (int w = 0; w < 8; ++w) s += red[comp * 32 + g0 + w];
            buf[comp * units + unit] = s;
        }
    }
}

// The K sums of the groups' component-major partials (publish_unit), in every thread of the block.  The tree is
// scene_sums_3g's: the G groups of 256 threads take components q, q + G, ...; thread lt adds units lt, lt + 256, ...
// in order (absent ones as +0.0), then the warp butterfly and the 8 warps in order.  unit_loads issues the loads of
// the thread's first U units (so that the caller can put them ahead of other memory traffic); unit_sums adds them,
// then any further units, and reduces.
template <int K, int G, int U>
__device__ __forceinline__ void unit_loads(const double* __restrict__ buf, int units, double (&v)[K][U]) {
    constexpr int KPT = (K + G - 1) / G;
    const int q = threadIdx.x >> 8, lt = threadIdx.x & 255;
#pragma unroll
    for (int j = 0; j < KPT; ++j)
#pragma unroll
        for (int u = 0; u < U; ++u)
            v[j][u] = q < G && q + G * j < K && lt + u * kThreads < units ? buf[(q + G * j) * units + lt + u * kThreads] : 0.0;
}

template <int K, int G, int U>
__device__ __forceinline__ void unit_sums(const double* __restrict__ buf, int units, const double (&v)[K][U],
                                          double (&tot)[K], double* red) {
    constexpr int KPT = (K + G - 1) / G;
    const int q = threadIdx.x >> 8, lt = threadIdx.x & 255;
    double acc[KPT];
#pragma unroll
    for (int j = 0; j < KPT; ++j) {
        acc[j] = 0.0;
#pragma unroll
        for (int u = 0; u < U; ++u) acc[j] += v[j][u];
    }
    if (q < G) {
        for (int c = lt + U * kThreads; c < units; c += kThreads) {
#pragma unroll
            for (int j = 0; j < KPT; ++j)
                if (q + G * j < K) acc[j] += buf[(q + G * j) * units + c];
        }
#pragma unroll
        for (int j = 0; j < KPT; ++j) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], o);
        }
    }
    const int lane = threadIdx.x & 31, wq = lt >> 5;
    __syncthreads();
    if (q < G && lane == 0) {
#pragma unroll
        for (int j = 0; j < KPT; ++j)
            if (q + G * j < K) red[(q + G * j) * 32 + wq] = acc[j];
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < K; ++c) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < kThreads / 32; ++w) s += red[c * 32 + w];
        tot[c] = s;
    }
}

// cell m (0..3) of thread lt in a tile
struct Cell {
    int t, i, j, k;
    bool ok;
};

__device__ __forceinline__ Cell tile_cell(const TileItem& ti, int n, int lt, int m) {
    Cell c;
    c.i = ti.i0 + m;
    c.j = ti.j0 + (lt >> 5);
    c.k = ti.k0 + (lt & 31);
    c.ok = c.i < n && c.j < n && c.k < n;
    c.t = (c.i * n + c.j) * n + c.k;
    return c;
}

// Search direction at cell t for iteration k: p_k = z + beta p_{k-1} (warp's _cg_kernel_2), or z at k = 1.
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

// The same two sums with every load hoisted, for the streaming kernel, where each thread's loads should all be in
// flight at once.  Every load is in bounds (a missing neighbour reads the cell itself, face fractions exist on all n+1 layers), so all
// of them can be in flight at once; the terms of domain faces are then left out of the sum, in the reference's order.
template <class X>
__device__ __forceinline__ float lap_acc_hoisted(const hf_scene& S, const X& x, float xc, int t, int i, int j, int k) {
    const int n = S.n, nn = n * n;
    const bool in0 = i > 0, in1 = i < n - 1, in2 = j > 0, in3 = j < n - 1, in4 = k > 0, in5 = k < n - 1;
    const float x0 = x(in0 ? t - nn : t), x1 = x(in1 ? t + nn : t), x2 = x(in2 ? t - n : t), x3 = x(in3 ? t + n : t),
                x4 = x(in4 ? t - 1 : t), x5 = x(in5 ? t + 1 : t);
    const float a0 = __ldg(S.ax + uidx_(n, i, j, k)), a1 = __ldg(S.ax + uidx_(n, i + 1, j, k)),
                a2 = __ldg(S.ay + vidx_(n, i, j, k)), a3 = __ldg(S.ay + vidx_(n, i, j + 1, k)),
                a4 = __ldg(S.az + widx_(n, i, j, k)), a5 = __ldg(S.az + widx_(n, i, j, k + 1));
    float acc = 0.0f;
    if (in0) acc = __fadd_rn(acc, __fmul_rn(a0, __fsub_rn(xc, x0)));
    if (in1) acc = __fadd_rn(acc, __fmul_rn(a1, __fsub_rn(xc, x1)));
    if (in2) acc = __fadd_rn(acc, __fmul_rn(a2, __fsub_rn(xc, x2)));
    if (in3) acc = __fadd_rn(acc, __fmul_rn(a3, __fsub_rn(xc, x3)));
    if (in4) acc = __fadd_rn(acc, __fmul_rn(a4, __fsub_rn(xc, x4)));
    if (in5) acc = __fadd_rn(acc, __fmul_rn(a5, __fsub_rn(xc, x5)));
    return acc;
}

// heat.py:55-91 neighbour_terms with use_fixed = 0; kappa_f from the precomputed face diffusivities (loads hoisted
// and kept in bounds as in lap_acc)
template <class X>
__device__ __forceinline__ float heat_nt_hoisted(const hf_scene& S, const X& x, float xc, int t, int i, int j, int k) {
    const int n = S.n, nn = n * n;
    const uint8_t* __restrict__ fl = S.cell_flags;
    const bool in[6] = {i > 0, i < n - 1, j > 0, j < n - 1, k > 0, k < n - 1};
    const int step[6] = {-nn, nn, -n, n, -1, 1};
    const int fidx[6] = {uidx_(n, i, j, k), uidx_(n, i + 1, j, k), vidx_(n, i, j, k), vidx_(n, i, j + 1, k),
                         widx_(n, i, j, k), widx_(n, i, j, k + 1)};
    const float* __restrict__ hk[3] = {S.hkx, S.hky, S.hkz};
    float xn[6], kf[6];
    uint8_t fn[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        const int nb = in[s] ? t + step[s] : t;
        xn[s] = x(nb);
        fn[s] = __ldg(fl + nb);
        kf[s] = __ldg(hk[s >> 1] + fidx[s]);
    }
    float acc = 0.0f;
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        if (!in[s]) continue;
        acc = __fadd_rn(acc, (fn[s] & 1) ? __fmul_rn(kf[s], xc) : __fmul_rn(kf[s], __fsub_rn(xc, xn[s])));
    }
    return acc;
}

// Set-up of one cell (heat.py:198-203 + k_heat_rhs/k_heat_diag; grid.py:238-248 mean removal + k_jacobi): returns
// b, D, r for x0 (the advected T, or the previous pressure).  Every load comes first and stays in bounds (a missing
// neighbour reads the cell itself), so they are in flight together; the sums then take the in-domain terms in the
// reference's order (heat.py:121-144 k_heat_diag and heat_nt, or k_jacobi's face-fraction sum and lap_acc).
template <bool HEAT>
__device__ __forceinline__ void setup_cell(const hf_scene& S, const float* x, float mean, float hh, float c_dt,
                                           const Cell& c, float& b, float& d, float& r) {
    const int n = S.n, nn = n * n, t = c.t, i = c.i, j = c.j, k = c.k;
    const bool in[6] = {i > 0, i < n - 1, j > 0, j < n - 1, k > 0, k < n - 1};
    const int step[6] = {-nn, nn, -n, n, -1, 1};
    const int fidx[6] = {uidx_(n, i, j, k), uidx_(n, i + 1, j, k), vidx_(n, i, j, k), vidx_(n, i, j + 1, k),
                         widx_(n, i, j, k), widx_(n, i, j, k + 1)};
    const float xc = x[t];
    float xn[6], kf[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) xn[s] = x[in[s] ? t + step[s] : t];
    if (HEAT) {
        const float* __restrict__ hk[3] = {S.hkx, S.hky, S.hkz};
        const uint8_t* __restrict__ fl = S.cell_flags;
        uint8_t fn[6];
#pragma unroll
        for (int s = 0; s < 6; ++s) {
            kf[s] = __ldg(hk[s >> 1] + fidx[s]);
            fn[s] = __ldg(fl + (in[s] ? t + step[s] : t));
        }
        b = S.hrhs[t];
        if (fl[t] & 1) {
            d = 1.0f;
            r = __fsub_rn(b, xc);
        } else {
            float sd = 0.0f, nt = 0.0f;
#pragma unroll
            for (int s = 0; s < 6; ++s)
                if (in[s]) sd = __fadd_rn(sd, kf[s]);
#pragma unroll
            for (int s = 0; s < 6; ++s) {
                if (!in[s]) continue;
                nt = __fadd_rn(nt, (fn[s] & 1) ? __fmul_rn(kf[s], xc) : __fmul_rn(kf[s], __fsub_rn(xc, xn[s])));
            }
            d = __fdiv_rn(1.0f, __fadd_rn(1.0f, __fmul_rn(c_dt, sd)));
            r = __fsub_rn(b, __fadd_rn(xc, __fmul_rn(c_dt, nt)));
        }
    } else {
        const float* __restrict__ af[3] = {S.ax, S.ay, S.az};
#pragma unroll
        for (int s = 0; s < 6; ++s) kf[s] = __ldg(af[s >> 1] + fidx[s]);
        b = S.rhs[t];
        if (mean != 0.0f) {
            b = __fsub_rn(b, mean);
            S.rhs[t] = b;
        }
        float sa = 0.0f, acc = 0.0f;
#pragma unroll
        for (int s = 0; s < 6; ++s)
            if (in[s]) sa = __fadd_rn(sa, kf[s]);
#pragma unroll
        for (int s = 0; s < 6; ++s)
            if (in[s]) acc = __fadd_rn(acc, __fmul_rn(kf[s], __fsub_rn(xc, xn[s])));
        d = __fdiv_rn(hh, maxf_(sa, 1.0e-12f));
        r = __fsub_rn(b, __fdiv_rn(acc, hh));
    }
}

// grid.py:140-153 k_project for the three low faces of a cell (and the high wall faces on the last layer)
__device__ __forceinline__ void project_cell(const hf_scene& S, float* u, float* v, float* w, const float* p, float pc,
                                             float dtr, float h, const Cell& c) {
    const int n = S.n, nn = n * n, t = c.t, i = c.i, j = c.j, k = c.k;
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

// Per-block copy of a scene's CG scalars; every block derives them from the same partial sums, so all copies agree.
struct LocalScene {
    double rz, atol_sq, bb, rr, pAp, mean;
    double true_rr;             // fp64 |b - A x|^2 of the outer defect correction (-1: not formed)
    float alpha, beta;
    int live, iters, maxit, status;
    int kbase;                  // iterations before the last restart by the defect correction
    int corrections;            // restarts so far
    int dc;                     // the true residual is still to be checked (HF_FLAG_DEFECT_CORRECTION)
};

__device__ __forceinline__ void init_scalars(LocalScene& L, const hf_scene& S, bool heat, const double (&tot)[3], int N) {
    const double tol = heat ? S.heat_tol : S.cg_tol;
    double atol = tol * sqrt(tot[0]);
    if (atol < tol) atol = tol;
    if (atol < 1.0e-18) atol = 1.0e-18;
    int maxit = heat ? S.heat_maxiter : S.cg_max_iter;
    if (maxit <= 0) maxit = N;
    L.maxit = maxit + (maxit & 1);   // iterations run in pairs
    L.bb = tot[0];
    L.rr = tot[1];
    L.rz = tot[2];
    L.atol_sq = atol * atol;
    L.iters = 0;
    L.beta = 0.0f;
    L.alpha = 0.0f;
    L.status = isfinite(tot[1]) ? 0 : HF_SCENE_NONFINITE;
    L.live = tot[1] > L.atol_sq && isfinite(tot[1]) && L.maxit > 0;
    L.true_rr = -1.0;
    L.kbase = 0;
    L.corrections = 0;
    L.dc = (S.flags & HF_FLAG_DEFECT_CORRECTION) != 0;
}

// convergence test after phase B of iteration kit (warp: kernel_2 then the residual test)
__device__ __forceinline__ bool update_scalars(LocalScene& L, bool heat, double rr, double rz, int kit) {
    L.iters = kit;
    const bool above = rr > L.atol_sq;
    L.beta = above ? __double2float_rn(rz / L.rz) : 0.0f;
    L.rz = rz;
    L.rr = rr;
    if (!isfinite(rr)) L.status |= HF_SCENE_NONFINITE;
    const bool live = above && isfinite(rr) && kit < L.maxit;
    if (!live && above && isfinite(rr)) L.status |= heat ? HF_SCENE_HEAT_MAXITER : HF_SCENE_PRESSURE_MAXITER;
    L.live = live;
    return live;
}

// True residual b - A x of one cell for the outer defect correction: the binary32 operator (grid.py:94-115 with the
// binary32 h^2; heat.py:94-105 with the binary32 dt/h^2 and face diffusivities) applied with every product and sum in
// fp64 to the binary32 vectors.
__device__ double true_residual_pressure(const hf_scene& S, const float* __restrict__ x, int t, int i, int j, int k,
                                         double hh) {
    const int n = S.n, nn = n * n;
    const double xc = x[t];
    double acc = 0.0;
    if (i > 0) acc += (double)S.ax[uidx_(n, i, j, k)] * (xc - (double)x[t - nn]);
    if (i < n - 1) acc += (double)S.ax[uidx_(n, i + 1, j, k)] * (xc - (double)x[t + nn]);
    if (j > 0) acc += (double)S.ay[vidx_(n, i, j, k)] * (xc - (double)x[t - n]);
    if (j < n - 1) acc += (double)S.ay[vidx_(n, i, j + 1, k)] * (xc - (double)x[t + n]);
    if (k > 0) acc += (double)S.az[widx_(n, i, j, k)] * (xc - (double)x[t - 1]);
    if (k < n - 1) acc += (double)S.az[widx_(n, i, j, k + 1)] * (xc - (double)x[t + 1]);
    return (double)S.rhs[t] - acc / hh;
}

__device__ double true_residual_heat(const hf_scene& S, const float* __restrict__ x, int t, int i, int j, int k,
                                     double c_dt) {
    const int n = S.n, nn = n * n;
    const double xc = x[t], b = S.hrhs[t];
    if (S.cell_flags[t] & 1) return b - xc;
    const int nbr[6] = {t - nn, t + nn, t - n, t + n, t - 1, t + 1};
    const bool in[6] = {i > 0, i < n - 1, j > 0, j < n - 1, k > 0, k < n - 1};
    const int fidx[6] = {uidx_(n, i, j, k), uidx_(n, i + 1, j, k), vidx_(n, i, j, k), vidx_(n, i, j + 1, k),
                         widx_(n, i, j, k), widx_(n, i, j, k + 1)};
    const float* hk[3] = {S.hkx, S.hky, S.hkz};
    double acc = 0.0;
    for (int q = 0; q < 6; ++q) {
        if (!in[q]) continue;
        const double kf = hk[q >> 1][fidx[q]];
        acc += (S.cell_flags[nbr[q]] & 1) ? kf * xc : kf * (xc - (double)x[nbr[q]]);
    }
    return b - (xc + c_dt * acc);
}

__device__ __forceinline__ void write_stats(const hf_scene& S, const LocalScene& L, bool heat, bool timed_out, int par) {
    hf_scene_state* st = S.state;
    if (heat) {
        st->status = L.status | (timed_out ? HF_SCENE_BARRIER_TIMEOUT : 0);
        st->heat_iters = L.iters;
        st->heat_rr = L.rr;
        st->heat_atol = sqrt(L.atol_sq);
        st->heat_bb = L.bb;
        st->heat_true_rr = L.true_rr;
        st->total_heat_iters += L.iters;
    } else {
        st->status |= L.status | (timed_out ? HF_SCENE_BARRIER_TIMEOUT : 0);
        st->pressure_iters = L.iters;
        st->pressure_rr = L.rr;
        st->pressure_atol = sqrt(L.atol_sq);
        st->pressure_bb = L.bb;
        st->pressure_true_rr = L.true_rr;
        st->rhs_mean = L.mean;
        st->total_pressure_iters += L.iters;
        if (!timed_out) {
            st->parity = par ^ 1;
            st->substeps += 1;
        }
    }
}

// ============================================================================================ TMA staging
// Box geometry of the tiled pressure stencil (elements, innermost k first), all at 16-byte aligned k origins:
//   z / p_old : k in [k0-4, k0+36), j in [j0-1, j0+9), i in [i0-1, i0+5)   (one-cell halo; k widened to alignment)
//   alpha_f x : k in [k0, k0+32),   j in [j0, j0+8),   i in [i0, i0+5)     (low faces of the tile + next i layer)
//   alpha_f y : k in [k0, k0+32),   j in [j0, j0+9),   i in [i0, i0+4)
//   alpha_f z : k in [k0, k0+36),   j in [j0, j0+8),   i in [i0, i0+4)
// Out-of-range elements are zero-filled by the copy engine and never used (domain faces are skipped).
constexpr int kBZ = 40 * 10 * 6, kBX = 32 * 8 * 5, kBY = 32 * 9 * 4, kBW = 36 * 8 * 4;
constexpr int kSlotFloats = 2 * kBZ + kBX + kBY + kBW;   // 8384 floats = 33,536 bytes (a multiple of 128)
// Heat system: the same z / p boxes; face diffusivities x (face lattice), y (face lattice: rows j0..j0+8 of (n, n+1, n))
// and z (cell-layout copy) in the face-fraction places; the cell flags (bytes) k in [k0-16, k0+48), j in [j0-1, j0+9),
// i in [i0-1, i0+5) -- 16-byte aligned k origin; the owner's and the neighbours' fixed bits.
constexpr int kBF = 64 * 10 * 6;                                   // bytes
constexpr int kHeatSlotFloats = kSlotFloats + kBF / 4;             // 9344 floats = 37,376 bytes (a multiple of 128)

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// The first 128-byte aligned float of the dynamic shared memory (TMA destinations), derived from raw by pointer
// arithmetic so that the compiler keeps the shared address space: a round trip through an integer would turn every
// access to the boxes into a generic load or store.
__device__ __forceinline__ float* align128_shared(float* raw) {
    return raw + ((128u - (smem_addr(raw) & 127u)) & 127u) / 4u;
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// bounded wait for the given phase; returns false on timeout
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned phase) {
    const unsigned long long t0 = global_timer_ns();
    for (unsigned spins = 0;; ++spins) {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(smem_addr(bar)), "r"(phase)
            : "memory");
        if (ok) return true;
        if ((spins & 63u) == 63u && global_timer_ns() - t0 > c_wait_limit_ns) return false;
    }
}

__device__ __forceinline__ void tma_load_3d(float* dst, const CUtensorMap* map, int x, int y, int z, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_addr(dst)), "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

// Tiles c = first, first + step, ... < end of scenes still iterating, through two shared-memory slots: the boxes of the
// next tile are requested (issue, thread 0) before the current tile is worked on, so the copy overlaps the work.  Bit s
// of ph is the phase the next wait on slot s expects.
// `work` must end with a __syncthreads after its last read of the slot (the slot is refilled next).  A wait that times
// out sets the error flag and waits once more for the copy, so that no copy is left in flight.
template <class Issue, class Work>
__device__ __forceinline__ void pipelined_tiles(int first, int end, int step, const LocalScene* loc, int scene_lo,
                                                const TileItem* __restrict__ tiles, float* slots,
                                                unsigned long long* mbar, unsigned& ph, int* err, Issue issue, Work work) {
    auto next_live = [&](int c) {
        while (c < end && !loc[tiles[c].scene - scene_lo].live) c += step;
        return c;
    };
    int cur = next_live(first), si = 0;
    if (cur < end && threadIdx.x == 0) issue(cur, slots, &mbar[0]);
    while (cur < end) {
        const int nxt = next_live(cur + step);
        if (nxt < end && threadIdx.x == 0) issue(nxt, slots + (si ^ 1) * kSlotFloats, &mbar[si ^ 1]);
        const unsigned phase = (ph >> si) & 1u;
        if (!mbar_wait(&mbar[si], phase)) {
            if (threadIdx.x == 0) atomicExch(err, 1);
            mbar_wait(&mbar[si], phase);
        }
        ph ^= 1u << si;
        work(cur, slots + si * kSlotFloats);
        cur = nxt;
        si ^= 1;
    }
}

// ================================================================================================== streaming
// A launch solves the groups of a GroupTable: consecutive scenes whose CG vectors the host sized to stay in L2.  The
// grid is split into gt.lanes lanes of equal size (lane = blockIdx.x / blocks per lane), each with its own barrier;
// a lane takes the next unsolved group from a queue counter, so independent groups run side by side and one lane's
// barrier waits overlap another lane's stencils on the same SM.  Inside a group, tiles are dealt round-robin over the
// lane's blocks (an equal share of every live scene per block while scenes converge at different iterations); every
// block sums the tile partials of every scene of the group itself (same bits everywhere) and keeps the scalars in
// shared memory, so an iteration takes two lane barriers.  Returns false when a barrier timed out.
template <bool HEAT, bool TMA>
__device__ bool solve_group(const hf_scene* __restrict__ scenes, const TileItem* __restrict__ tiles, const int4 grp,
                            int lb, int nlb, unsigned* bar, unsigned& epoch, double dt_d, const Workspace& ws,
                            double* red, LocalScene* loc, unsigned char* s_par, int* s_any, float* slots,
                            unsigned long long* mbar, unsigned& ph) {
    const int scene_lo = grp.x, scene_hi = grp.y, tile_lo = grp.z, tile_hi = grp.w;
    const int ns = scene_hi - scene_lo;
    double* bufA = ws.partA;
    double* bufB = ws.partB;
    const float dt = (float)dt_d;
    const int lt = threadIdx.x;
    const int first = tile_lo + lb;
    bool ok = true;
    if (threadIdx.x < ns) s_par[threadIdx.x] = (unsigned char)scenes[scene_lo + threadIdx.x].state->parity;

    // ---------------------------------------------------------------------------------------- prologue
    for (int q = 0; q < ns; ++q) {
        const int s = scene_lo + q;
        if (!HEAT) {
            // the pressure rhs mean (grid.py:238-241) from the divergence stage's chunk sums
            double m[1];
            const int comp[1] = {0};
            scene_sums<1>(ws.mean_part, ws.chunk_begin[s], ws.chunk_begin[s + 1], comp, m, red, 0);
            const int n = scenes[s].n;
            if (threadIdx.x == 0) loc[q].mean = (double)__double2float_rn(m[0] / ((double)n * n * n));
        } else if (threadIdx.x == 0) {
            loc[q].mean = 0.0;
        }
    }
    __syncthreads();
    for (int c = first; c < tile_hi; c += nlb) {
        const TileItem ti = tiles[c];
        const hf_scene& S = scenes[ti.scene];
        const int n = S.n, par = s_par[ti.scene - scene_lo];
        const float h = (float)S.h, hh = __fmul_rn(h, h), c_dt = __fdiv_rn(dt, hh);
        const float* x = HEAT ? S.T[par ^ 1] : S.p;
        const float mean = (float)loc[ti.scene - scene_lo].mean;
        double part[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const Cell cl = tile_cell(ti, n, lt, m);
            if (!cl.ok) continue;
            float b, d, r;
            setup_cell<HEAT>(S, x, mean, hh, c_dt, cl, b, d, r);
            const float z = __fmul_rn(d, r);
            (HEAT ? S.hdiag : S.pdiag)[cl.t] = d;
            S.cg_r[cl.t] = r;
            S.cg_z[cl.t] = z;
            part[0] += (double)b * (double)b;
            part[1] += (double)r * (double)r;
            part[2] += (double)r * (double)z;
        }
        group_sum<3>(part, red);
        if (lt == 0) {
            bufB[c] = part[0];
            bufB[1 * ws.tiles + c] = part[1];
            bufB[2 * ws.tiles + c] = part[2];
        }
    }
    if (!(ok = grid_barrier(bar, epoch, ws.err, nlb))) goto done;
    for (int q = 0; q < ns; ++q) {
        const int s = scene_lo + q;
        const int b = ws.tile_begin[s], e = ws.tile_begin[s + 1];
        double tot[3];
        const int comp[3] = {0, 1, 2};
        scene_sums<3>(bufB, b, e, comp, tot, red, ws.tiles);
        if (threadIdx.x == 0) {
            const hf_scene& S = scenes[s];
            const double mean = loc[q].mean;
            init_scalars(loc[q], S, HEAT, tot, S.n * S.n * S.n);
            loc[q].mean = mean;
            loc[q].live = loc[q].live && b < e;
        }
    }
    if (threadIdx.x == 0) {
        int any = 0;
        for (int q = 0; q < ns; ++q) any |= loc[q].live;
        *s_any = any;
    }
    __syncthreads();

    // ------------------------------------------------------------------------------------------ iterations
    // Rounds: CG iterations until every scene has stopped; then, for scenes with the outer defect correction, the true
    // residual, and another round for the scenes it restarted.
    for (;;) {
    for (int kit = 1; *s_any; ++kit) {
        // phase A: p_k at the stencil points, Ap = A p_k, p.Ap
        if constexpr (TMA) {
            // stage z and p_{k-1} with a one-cell halo and the tile's face fractions (the resident kernel's box
            // geometry), form p_k in place, A p from shared memory
            const bool first_it = kit == 1;
            auto issue = [&](int c, float* slot, unsigned long long* mb) {
                const TileItem ti = tiles[c];
                asm volatile("fence.proxy.async.global;" ::: "memory");
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                const bool go = *(volatile int*)ws.err == 0;
                const CUtensorMap* M = ws.maps + kMapsPerScene * ti.scene;
                mbar_expect_tx(mb, go ? (unsigned)(((first_it ? 1 : 2) * kBZ + kBX + kBY + kBW) * sizeof(float)) : 0u);
                if (go) {
                    tma_load_3d(slot, &M[0], ti.k0 - 4, ti.j0 - 1, ti.i0 - 1, mb);
                    if (!first_it) tma_load_3d(slot + kBZ, &M[1 + ((kit - 1) & 1)], ti.k0 - 4, ti.j0 - 1, ti.i0 - 1, mb);
                    tma_load_3d(slot + 2 * kBZ, &M[3], ti.k0, ti.j0, ti.i0, mb);
                    tma_load_3d(slot + 2 * kBZ + kBX, &M[4], ti.k0, ti.j0, ti.i0, mb);
                    tma_load_3d(slot + 2 * kBZ + kBX + kBY, &M[5], ti.k0, ti.j0, ti.i0, mb);
                }
            };
            auto work = [&](int c, float* slot) {
                const TileItem ti = tiles[c];
                const LocalScene& L = loc[ti.scene - scene_lo];
                const hf_scene& S = scenes[ti.scene];
                const int n = S.n;
                const float h = (float)S.h, hh = __fmul_rn(h, h);
                if (!first_it)
                    for (int e = lt; e < kBZ; e += kThreads) slot[e] = __fadd_rn(slot[e], __fmul_rn(L.beta, slot[kBZ + e]));
                __syncthreads();
                const float* axb = slot + 2 * kBZ;
                const float* ayb = axb + kBX;
                const float* azb = ayb + kBY;
                float* pnew = S.cg_p[kit & 1];
                double part[1] = {0.0};
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                    const Cell cl = tile_cell(ti, n, lt, m);
                    if (!cl.ok) continue;
                    const int bi = m, bj = lt >> 5, bk = lt & 31;
                    const int o = (bi + 1) * 400 + (bj + 1) * 40 + (bk + 4);
                    const float pc = slot[o];
                    float acc = 0.0f;
                    if (cl.i > 0) acc = __fadd_rn(acc, __fmul_rn(axb[bi * 256 + bj * 32 + bk], __fsub_rn(pc, slot[o - 400])));
                    if (cl.i < n - 1)
                        acc = __fadd_rn(acc, __fmul_rn(axb[(bi + 1) * 256 + bj * 32 + bk], __fsub_rn(pc, slot[o + 400])));
                    if (cl.j > 0) acc = __fadd_rn(acc, __fmul_rn(ayb[bi * 288 + bj * 32 + bk], __fsub_rn(pc, slot[o - 40])));
                    if (cl.j < n - 1)
                        acc = __fadd_rn(acc, __fmul_rn(ayb[bi * 288 + (bj + 1) * 32 + bk], __fsub_rn(pc, slot[o + 40])));
                    if (cl.k > 0) acc = __fadd_rn(acc, __fmul_rn(azb[bi * 288 + bj * 36 + bk], __fsub_rn(pc, slot[o - 1])));
                    if (cl.k < n - 1)
                        acc = __fadd_rn(acc, __fmul_rn(azb[bi * 288 + bj * 36 + bk + 1], __fsub_rn(pc, slot[o + 1])));
                    const float ap = __fdiv_rn(acc, hh);
                    pnew[cl.t] = pc;
                    S.cg_Ap[cl.t] = ap;
                    part[0] += (double)pc * (double)ap;
                }
                group_sum<1>(part, red);   // its __syncthreads also ends every read of the slot
                if (lt == 0) bufA[c] = part[0];
            };
            pipelined_tiles(first, tile_hi, nlb, loc, scene_lo, tiles, slots, mbar, ph, ws.err, issue, work);
        }
        for (int c = first; !TMA && c < tile_hi; c += nlb) {
            const TileItem ti = tiles[c];
            const LocalScene& L = loc[ti.scene - scene_lo];
            if (!L.live) continue;
            const hf_scene& S = scenes[ti.scene];
            const int n = S.n;
            const float h = (float)S.h, hh = __fmul_rn(h, h), c_dt = __fdiv_rn(dt, hh);
            const Dir P{S.cg_z, S.cg_p[(kit - 1) & 1], L.beta, kit == 1};
            float pc[4], ap[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const Cell cl = tile_cell(ti, n, lt, m);
                pc[m] = ap[m] = 0.0f;
                if (!cl.ok) continue;
                pc[m] = P(cl.t);
                if (HEAT) {
                    ap[m] = (__ldg(S.cell_flags + cl.t) & 1)
                                ? pc[m]
                                : __fadd_rn(pc[m], __fmul_rn(c_dt, heat_nt_hoisted(S, P, pc[m], cl.t, cl.i, cl.j, cl.k)));
                } else {
                    ap[m] = __fdiv_rn(lap_acc_hoisted(S, P, pc[m], cl.t, cl.i, cl.j, cl.k), hh);
                }
            }
            float* pnew = S.cg_p[kit & 1];
            double part[1] = {0.0};
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const Cell cl = tile_cell(ti, n, lt, m);
                if (!cl.ok) continue;
                pnew[cl.t] = pc[m];
                S.cg_Ap[cl.t] = ap[m];
                part[0] += (double)pc[m] * (double)ap[m];
            }
            group_sum<1>(part, red);
            if (lt == 0) bufA[c] = part[0];
        }
        if (!(ok = grid_barrier(bar, epoch, ws.err, nlb))) goto done;
        {
            // every live scene's p.Ap (live: shared values written before the last __syncthreads)
            const int comp[1] = {0};
            group_sums<1>(bufA, ws.tile_begin, scene_lo, ns, comp, ws.tiles, red, [&](int q) { return (bool)loc[q].live; },
                          [&](int q, const double(&tot)[1]) {
                              loc[q].pAp = tot[0];
                              loc[q].alpha = __double2float_rn(loc[q].rz / tot[0]);
                          });
        }
        // phase B: x += alpha p, r -= alpha Ap, z = D r, r.r and r.z
        if constexpr (TMA) {
            // the tile's x, p_k, r, Ap and D as five (32, 8, 4) boxes: element (m, lt / 32, lt % 32) at m 256 + lt
            auto issue = [&](int c, float* slot, unsigned long long* mb) {
                const TileItem ti = tiles[c];
                asm volatile("fence.proxy.async.global;" ::: "memory");
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                const bool go = *(volatile int*)ws.err == 0;
                const CUtensorMap* M = ws.maps + kMapsPerScene * ti.scene;
                mbar_expect_tx(mb, go ? (unsigned)(5 * 1024 * sizeof(float)) : 0u);
                if (go) {
                    tma_load_3d(slot, &M[6], ti.k0, ti.j0, ti.i0, mb);
                    tma_load_3d(slot + 1024, &M[7 + (kit & 1)], ti.k0, ti.j0, ti.i0, mb);
                    tma_load_3d(slot + 2048, &M[9], ti.k0, ti.j0, ti.i0, mb);
                    tma_load_3d(slot + 3072, &M[10], ti.k0, ti.j0, ti.i0, mb);
                    tma_load_3d(slot + 4096, &M[11], ti.k0, ti.j0, ti.i0, mb);
                }
            };
            auto work = [&](int c, float* slot) {
                const TileItem ti = tiles[c];
                const LocalScene& L = loc[ti.scene - scene_lo];
                const hf_scene& S = scenes[ti.scene];
                const int n = S.n;
                const float alpha = L.alpha;
                double part[2] = {0.0, 0.0};
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                    const Cell cl = tile_cell(ti, n, lt, m);
                    if (!cl.ok) continue;
                    const int e = m * 256 + lt;
                    const float xv = __fadd_rn(slot[e], __fmul_rn(alpha, slot[1024 + e]));
                    const float rv = __fsub_rn(slot[2048 + e], __fmul_rn(alpha, slot[3072 + e]));
                    const float zv = __fmul_rn(slot[4096 + e], rv);
                    S.p[cl.t] = xv;
                    S.cg_r[cl.t] = rv;
                    S.cg_z[cl.t] = zv;
                    part[0] += (double)rv * (double)rv;
                    part[1] += (double)rv * (double)zv;
                }
                group_sum<2>(part, red);
                if (lt == 0) {
                    bufB[1 * ws.tiles + c] = part[0];
                    bufB[2 * ws.tiles + c] = part[1];
                }
            };
            pipelined_tiles(first, tile_hi, nlb, loc, scene_lo, tiles, slots, mbar, ph, ws.err, issue, work);
        }
        for (int c = first; !TMA && c < tile_hi; c += nlb) {
            const TileItem ti = tiles[c];
            const LocalScene& L = loc[ti.scene - scene_lo];
            if (!L.live) continue;
            const hf_scene& S = scenes[ti.scene];
            const int n = S.n, par = s_par[ti.scene - scene_lo];
            float* x = HEAT ? S.T[par ^ 1] : S.p;
            const float* D = HEAT ? S.hdiag : S.pdiag;
            const float* pk = S.cg_p[kit & 1];
            const float alpha = L.alpha;
            float xv[4], rv[4], zv[4];
            {
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                    const Cell cl = tile_cell(ti, n, lt, m);
                    xv[m] = rv[m] = zv[m] = 0.0f;
                    if (!cl.ok) continue;
                    xv[m] = __fadd_rn(x[cl.t], __fmul_rn(alpha, pk[cl.t]));
                    rv[m] = __fsub_rn(S.cg_r[cl.t], __fmul_rn(alpha, S.cg_Ap[cl.t]));
                    zv[m] = __fmul_rn(D[cl.t], rv[m]);
                }
            }
            double part[2] = {0.0, 0.0};
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const Cell cl = tile_cell(ti, n, lt, m);
                if (!cl.ok) continue;
                x[cl.t] = xv[m];
                S.cg_r[cl.t] = rv[m];
                S.cg_z[cl.t] = zv[m];
                part[0] += (double)rv[m] * (double)rv[m];
                part[1] += (double)rv[m] * (double)zv[m];
            }
            group_sum<2>(part, red);
            if (lt == 0) {
                bufB[1 * ws.tiles + c] = part[0];
                bufB[2 * ws.tiles + c] = part[1];
            }
        }
        if (!(ok = grid_barrier(bar, epoch, ws.err, nlb))) goto done;
        {
            // every live scene's r.r and r.z, then its convergence test
            const int comp[2] = {1, 2};
            group_sums<2>(bufB, ws.tile_begin, scene_lo, ns, comp, ws.tiles, red, [&](int q) { return (bool)loc[q].live; },
                          [&](int q, const double(&tot)[2]) { update_scalars(loc[q], HEAT, tot[0], tot[1], loc[q].kbase + kit); });
        }
        if (threadIdx.x == 0) {
            int any = 0;
            for (int q = 0; q < ns; ++q) any |= loc[q].live;
            *s_any = any;
        }
        __syncthreads();
    }
    // ------------------------------------------------------------- outer defect correction (fp64 true residual)
    if (threadIdx.x == 0) {
        int any = 0;
        for (int q = 0; q < ns; ++q) any |= loc[q].dc;
        *s_any = any;
    }
    __syncthreads();
    if (!*s_any) break;
    // pass 1: r_true = b - A x in fp64 for the scenes to check, rounded into the Ap vector (free between solves)
    for (int c = first; c < tile_hi; c += nlb) {
        const TileItem ti = tiles[c];
        if (!loc[ti.scene - scene_lo].dc) continue;
        const hf_scene& S = scenes[ti.scene];
        const int n = S.n, par = s_par[ti.scene - scene_lo];
        const float h = (float)S.h, hh = __fmul_rn(h, h), c_dt = __fdiv_rn(dt, hh);
        const float* x = HEAT ? S.T[par ^ 1] : S.p;
        double part[1] = {0.0};
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const Cell cl = tile_cell(ti, n, lt, m);
            if (!cl.ok) continue;
            const double rt = HEAT ? true_residual_heat(S, x, cl.t, cl.i, cl.j, cl.k, (double)c_dt)
                                   : true_residual_pressure(S, x, cl.t, cl.i, cl.j, cl.k, (double)hh);
            S.cg_Ap[cl.t] = __double2float_rn(rt);
            part[0] += rt * rt;
        }
        group_sum<1>(part, red);
        if (lt == 0) bufA[1 * ws.tiles + c] = part[0];
    }
    if (!(ok = grid_barrier(bar, epoch, ws.err, nlb))) goto done;
    for (int q = 0; q < ns; ++q) {
        if (!loc[q].dc) continue;   // uniform: shared value
        const int s = scene_lo + q;
        double tot[1];
        const int comp[1] = {1};
        scene_sums<1>(bufA, ws.tile_begin[s], ws.tile_begin[s + 1], comp, tot, red, ws.tiles);
        if (threadIdx.x == 0) {
            LocalScene& L = loc[q];
            L.true_rr = tot[0];
            // restart from x with the true residual when it is above the tolerance, the recurrence had converged
            // (not stopped at maxiter or on a non-finite value) and corrections are left
            const bool stopped = L.status & (HF_SCENE_NONFINITE | HF_SCENE_HEAT_MAXITER | HF_SCENE_PRESSURE_MAXITER);
            L.live = isfinite(tot[0]) && tot[0] > L.atol_sq && !stopped && L.corrections < kMaxCorrections &&
                     L.iters < L.maxit;
            L.dc = L.live;
            if (L.live) {
                L.corrections += 1;
                L.status |= HF_SCENE_CORRECTED;
                L.kbase = L.iters;
            }
        }
    }
    if (threadIdx.x == 0) {
        int any = 0;
        for (int q = 0; q < ns; ++q) any |= loc[q].live;
        *s_any = any;
    }
    __syncthreads();
    if (!*s_any) break;
    // pass 2: r = r_true, z = D r for the restarted scenes; r.r and r.z start the next round (p_1 = z)
    for (int c = first; c < tile_hi; c += nlb) {
        const TileItem ti = tiles[c];
        if (!loc[ti.scene - scene_lo].live) continue;
        const hf_scene& S = scenes[ti.scene];
        const int n = S.n;
        const float* D = HEAT ? S.hdiag : S.pdiag;
        double part[2] = {0.0, 0.0};
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const Cell cl = tile_cell(ti, n, lt, m);
            if (!cl.ok) continue;
            const float r = S.cg_Ap[cl.t];
            const float z = __fmul_rn(D[cl.t], r);
            S.cg_r[cl.t] = r;
            S.cg_z[cl.t] = z;
            part[0] += (double)r * (double)r;
            part[1] += (double)r * (double)z;
        }
        group_sum<2>(part, red);
        if (lt == 0) {
            bufB[1 * ws.tiles + c] = part[0];
            bufB[2 * ws.tiles + c] = part[1];
        }
    }
    if (!(ok = grid_barrier(bar, epoch, ws.err, nlb))) goto done;
    for (int q = 0; q < ns; ++q) {
        if (!loc[q].live) continue;
        const int s = scene_lo + q;
        double tot[2];
        const int comp[2] = {1, 2};
        scene_sums<2>(bufB, ws.tile_begin[s], ws.tile_begin[s + 1], comp, tot, red, ws.tiles);
        if (threadIdx.x == 0) {
            LocalScene& L = loc[q];
            L.rr = tot[0];
            L.rz = tot[1];
            L.beta = 0.0f;
            L.live = isfinite(tot[0]) && tot[0] > L.atol_sq;
        }
    }
    if (threadIdx.x == 0) {
        int any = 0;
        for (int q = 0; q < ns; ++q) any |= loc[q].live;
        *s_any = any;
    }
    __syncthreads();
    }   // rounds
    // -------------------------------------------------------------------- pressure epilogue: projection
    if (!HEAT) {
        for (int c = first; c < tile_hi; c += nlb) {
            const TileItem ti = tiles[c];
            const hf_scene& S = scenes[ti.scene];
            const int n = S.n, par = s_par[ti.scene - scene_lo];
            const float h = (float)S.h, dtr = (float)(dt_d / S.rho);
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const Cell cl = tile_cell(ti, n, lt, m);
                if (cl.ok) project_cell(S, S.u[par ^ 1], S.v[par ^ 1], S.w[par ^ 1], S.p, S.p[cl.t], dtr, h, cl);
            }
        }
    }
done:
    // Every block of the lane read the group's parities before its first barrier, so the lane's first block may
    // flip them now (the lane's other blocks may already be in the next group: other scenes).
    __syncthreads();
    if (lb == 0) {
        for (int q = threadIdx.x; q < ns; q += kThreads) {
            const hf_scene& S = scenes[scene_lo + q];
            if (S.flags & HF_FLAG_ACTIVE) write_stats(S, loc[q], HEAT, !ok, s_par[q]);
        }
    }
    __syncthreads();
    return ok;
}

template <bool HEAT, bool TMA>
__global__ void __launch_bounds__(kThreads) k_pcg(const hf_scene* __restrict__ scenes, const TileItem* __restrict__ tiles,
                                                 double dt_d, Workspace ws, const __grid_constant__ GroupTable gt) {
    __shared__ double red[kRedComps * 32];
    __shared__ LocalScene loc[kGroupScenes];
    __shared__ unsigned char s_par[kGroupScenes];
    __shared__ int s_any;
    __shared__ __align__(8) unsigned long long mbar[2];
    extern __shared__ __align__(128) float sm_raw[];
    float* slots = TMA ? align128_shared(sm_raw) : nullptr;
    unsigned ph = 0u;   // bit s: the phase the next wait on slot s's mbarrier expects (a register, not an array)
    if (TMA && threadIdx.x == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int nlb = gridDim.x / gt.lanes;           // blocks per lane (the host launches a multiple of gt.lanes)
    const int lane = blockIdx.x / nlb, lb = blockIdx.x % nlb;
    unsigned* bar = ws.bar + (HEAT ? 0 : kMaxLanes) + lane;
    int* next = ws.lane_next + (HEAT ? 0 : kMaxLanes) + lane;
    unsigned* queue = ws.queue + (HEAT ? 0 : 1);
    unsigned epoch = 0;
    for (;;) {
        if (lb == 0 && threadIdx.x == 0) *(volatile int*)next = (int)atomicAdd(queue, 1u);
        if (!grid_barrier(bar, epoch, ws.err, nlb)) break;
        const int g = *(volatile int*)next;
        if (g >= gt.count) break;
        if (!solve_group<HEAT, TMA>(scenes, tiles, gt.g[g], lb, nlb, bar, epoch, dt_d, ws, red, loc, s_par, &s_any, slots,
                                    mbar, ph))
            break;
    }
    // a timed-out barrier leaves the groups that no lane reached unsolved: flag their scenes
    if (blockIdx.x == 0 && *(volatile int*)ws.err) {
        for (int q = 0; q < gt.count; ++q)
            for (int s = gt.g[q].x + (int)threadIdx.x; s < gt.g[q].y; s += kThreads)
                if (scenes[s].flags & HF_FLAG_ACTIVE) scenes[s].state->status |= HF_SCENE_BARRIER_TIMEOUT;
    }
}

// ======================================================================================= register-resident
// Block = `groups` x 256 threads; group g owns tiles c0 + g + groups*q (q < MAXC) of the block's contiguous range.
template <bool HEAT, int MAXC, bool TMA>
__global__ void __launch_bounds__(MAXC == 1 ? 1024 : (MAXC == 2 ? 768 : 512), 1)
    k_pcg_res(const hf_scene* __restrict__ scenes, const TileItem* __restrict__ tiles, int tile_lo, int tile_hi,
              double dt_d, Workspace ws, const __grid_constant__ TileMaps maps) {
    constexpr int CPT = 4 * MAXC;   // cells per thread
    extern __shared__ __align__(128) float sm_raw[];
    // TMA destinations must be 128-byte aligned: the launch adds 128 bytes of slack
    float* sm_boxes = align128_shared(sm_raw);
    __shared__ double red[kRedComps * 32];
    __shared__ LocalScene Ls;
    __shared__ __align__(8) unsigned long long mbar[4 * 3];
    __shared__ TileItem my_s[4 * 3];
    const int groups = blockDim.x >> 8, g = threadIdx.x >> 8, lt = threadIdx.x & 255;
    const int c0 = tile_lo + (int)(((long long)(tile_hi - tile_lo) * blockIdx.x) / gridDim.x);
    const int c1 = tile_lo + (int)(((long long)(tile_hi - tile_lo) * (blockIdx.x + 1)) / gridDim.x);
    const int sidx = tiles[c0].scene;   // one scene per plan on this path
    const hf_scene& S = scenes[sidx];
    const int n = S.n, N = n * n * n;
    const int par = S.state->parity;
    unsigned* bar = ws.bar + (HEAT ? 0 : kMaxLanes);
    unsigned epoch = 0;
    const float dt = (float)dt_d;
    const float h = (float)S.h, hh = __fmul_rn(h, h), c_dt = __fdiv_rn(dt, hh);
    double* bufA = ws.partA;
    double* bufB = ws.partB;
    const int cb = ws.tile_begin[sidx], ce = ws.tile_begin[sidx + 1];
    float* xg = HEAT ? S.T[par ^ 1] : S.p;
    float* zg = S.cg_z;
    // the group's tiles in shared memory (registers held through the solve make the stencil phases spill)
    TileItem* const my = my_s + g * MAXC;
    bool have[MAXC];
#pragma unroll
    for (int q = 0; q < MAXC; ++q) have[q] = c0 + g + groups * q < c1;
    if (lt < MAXC) {
        const int c = c0 + g + groups * lt;
        my[lt] = tiles[c < c1 ? c : c0];
    }
    unsigned phase_bit = 0;
    if (TMA && lt == 0) {
#pragma unroll
        for (int q = 0; q < MAXC; ++q) mbar_init(&mbar[g * MAXC + q], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    float x[CPT], r[CPT], z[CPT], p[CPT], D[CPT], Ap[CPT];
    // ------------------------------------------------------------------ prologue (values kept in registers)
    float mean = 0.0f;
    if (!HEAT) {
        double mm[1];
        const int comp[1] = {0};
        scene_sums<1>(ws.mean_part, ws.chunk_begin[sidx], ws.chunk_begin[sidx + 1], comp, mm, red, 0);
        mean = __double2float_rn(mm[0] / ((double)n * n * n));
    }
#pragma unroll
    for (int q = 0; q < MAXC; ++q) {
        double part[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const int s = q * 4 + m;
            x[s] = r[s] = z[s] = p[s] = D[s] = Ap[s] = 0.0f;
            const Cell cl = tile_cell(my[q], n, lt, m);
            if (!have[q] || !cl.ok) continue;
            float b, d, rr;
            setup_cell<HEAT>(S, xg, mean, hh, c_dt, cl, b, d, rr);
            x[s] = xg[cl.t];
            D[s] = d;
            r[s] = rr;
            z[s] = __fmul_rn(d, rr);
            zg[cl.t] = z[s];
            part[0] += (double)b * (double)b;
            part[1] += (double)rr * (double)rr;
            part[2] += (double)rr * (double)z[s];
        }
        group_sum<3>(part, red);
        const int c = c0 + g + groups * q;
        if (lt == 0 && have[q]) {
            bufB[c] = part[0];
            bufB[1 * ws.tiles + c] = part[1];
            bufB[2 * ws.tiles + c] = part[2];
        }
    }
    // the face fractions of the tiles stay in shared memory for the whole solve
    if (TMA && lt == 0) {
#pragma unroll
        for (int q = 0; q < MAXC; ++q) {
            if (!have[q]) continue;
            float* slot = sm_boxes + (size_t)(g * MAXC + q) * kSlotFloats;
            unsigned long long* mb = &mbar[g * MAXC + q];
            mbar_expect_tx(mb, (unsigned)((kBX + kBY + kBW) * sizeof(float)));
            tma_load_3d(slot + 2 * kBZ, &maps.ax, my[q].k0, my[q].j0, my[q].i0, mb);
            tma_load_3d(slot + 2 * kBZ + kBX, &maps.ayc, my[q].k0, my[q].j0, my[q].i0, mb);
            tma_load_3d(slot + 2 * kBZ + kBX + kBY, &maps.azc, my[q].k0, my[q].j0, my[q].i0, mb);
        }
    }
    if (TMA) {
        bool ok = true;
#pragma unroll
        for (int q = 0; q < MAXC; ++q)
            if (have[q]) ok = mbar_wait(&mbar[g * MAXC + q], phase_bit) && ok;
        if (!ok) atomicExch(ws.err, 1);
        phase_bit ^= 1u;
    }
    if (!grid_barrier(bar, epoch, ws.err, gridDim.x)) goto finish;
    {
        double tot[3];
        const int comp[3] = {0, 1, 2};
        scene_sums<3>(bufB, cb, ce, comp, tot, red, ws.tiles);
        if (threadIdx.x == 0) {
            init_scalars(Ls, S, HEAT, tot, N);
            Ls.mean = (double)mean;
        }
        __syncthreads();
    }
    // ------------------------------------------------------------------------------------------ iterations
    for (int kit = 1; Ls.live; ++kit) {
        // phase A: p_k, Ap = A p_k, p.Ap
        const float beta = Ls.beta;
        const bool first = kit == 1;
        const float* pold = S.cg_p[(kit - 1) & 1];
        float* pnew = S.cg_p[kit & 1];
        if (TMA) {
            // stage z and p_{k-1} (with halo) of every tile of the group, then form p_k in place over the z box
            if (lt == 0) {
                asm volatile("fence.proxy.async.global;" ::: "memory");
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
#pragma unroll
                for (int q = 0; q < MAXC; ++q) {
                    if (!have[q]) continue;
                    float* slot = sm_boxes + (size_t)(g * MAXC + q) * kSlotFloats;
                    unsigned long long* mb = &mbar[g * MAXC + q];
                    mbar_expect_tx(mb, (unsigned)((first ? 1 : 2) * kBZ * sizeof(float)));
                    tma_load_3d(slot, &maps.z, my[q].k0 - 4, my[q].j0 - 1, my[q].i0 - 1, mb);
                    if (!first)
                        tma_load_3d(slot + kBZ, ((kit - 1) & 1) ? &maps.p1 : &maps.p0, my[q].k0 - 4, my[q].j0 - 1,
                                    my[q].i0 - 1, mb);
                }
            }
            bool ok = true;
#pragma unroll
            for (int q = 0; q < MAXC; ++q)
                if (have[q]) ok = mbar_wait(&mbar[g * MAXC + q], phase_bit) && ok;
            if (!ok) atomicExch(ws.err, 1);
            phase_bit ^= 1u;
            if (!first) {
#pragma unroll
                for (int q = 0; q < MAXC; ++q) {
                    if (!have[q]) continue;
                    float* slot = sm_boxes + (size_t)(g * MAXC + q) * kSlotFloats;
                    for (int e = lt; e < kBZ; e += 256) slot[e] = __fadd_rn(slot[e], __fmul_rn(beta, slot[kBZ + e]));
                }
            }
            asm volatile("bar.sync %0, 256;" ::"r"(g + 1) : "memory");
#pragma unroll
            for (int q = 0; q < MAXC; ++q) {
                const float* slot = sm_boxes + (size_t)(g * MAXC + q) * kSlotFloats;
                const float* Pb = slot;
                const float* axb = slot + 2 * kBZ;
                const float* ayb = axb + kBX;
                const float* azb = ayb + kBY;
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                    const int s = q * 4 + m;
                    const Cell cl = tile_cell(my[q], n, lt, m);
                    if (!have[q] || !cl.ok) continue;
                    const float pc = first ? z[s] : __fadd_rn(z[s], __fmul_rn(beta, p[s]));
                    const int bi = cl.i - my[q].i0, bj = cl.j - my[q].j0, bk = cl.k - my[q].k0;
                    const int o = (bi + 1) * 400 + (bj + 1) * 40 + (bk + 4);
                    float acc = 0.0f;
                    if (cl.i > 0) acc = __fadd_rn(acc, __fmul_rn(axb[bi * 256 + bj * 32 + bk], __fsub_rn(pc, Pb[o - 400])));
                    if (cl.i < n - 1)
                        acc = __fadd_rn(acc, __fmul_rn(axb[(bi + 1) * 256 + bj * 32 + bk], __fsub_rn(pc, Pb[o + 400])));
                    if (cl.j > 0) acc = __fadd_rn(acc, __fmul_rn(ayb[bi * 288 + bj * 32 + bk], __fsub_rn(pc, Pb[o - 40])));
                    if (cl.j < n - 1)
                        acc = __fadd_rn(acc, __fmul_rn(ayb[bi * 288 + (bj + 1) * 32 + bk], __fsub_rn(pc, Pb[o + 40])));
                    if (cl.k > 0) acc = __fadd_rn(acc, __fmul_rn(azb[bi * 288 + bj * 36 + bk], __fsub_rn(pc, Pb[o - 1])));
                    if (cl.k < n - 1)
                        acc = __fadd_rn(acc, __fmul_rn(azb[bi * 288 + bj * 36 + bk + 1], __fsub_rn(pc, Pb[o + 1])));
                    Ap[s] = __fdiv_rn(acc, hh);
                    p[s] = pc;
                }
            }
        } else {
            const Dir P{zg, pold, beta, first};
#pragma unroll
            for (int q = 0; q < MAXC; ++q) {
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                    const int s = q * 4 + m;
                    const Cell cl = tile_cell(my[q], n, lt, m);
                    if (!have[q] || !cl.ok) continue;
                    const float pc = first ? z[s] : __fadd_rn(z[s], __fmul_rn(beta, p[s]));
                    if (HEAT) {
                        Ap[s] = (__ldg(S.cell_flags + cl.t) & 1)
                                    ? pc
                                    : __fadd_rn(pc, __fmul_rn(c_dt, heat_nt(S, P, pc, cl.t, cl.i, cl.j, cl.k)));
                    } else {
                        Ap[s] = __fdiv_rn(lap_acc(S, P, pc, cl.t, cl.i, cl.j, cl.k), hh);
                    }
                    p[s] = pc;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < MAXC; ++q) {
            double part[1] = {0.0};
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const int s = q * 4 + m;
                const Cell cl = tile_cell(my[q], n, lt, m);
                if (!have[q] || !cl.ok) continue;
                pnew[cl.t] = p[s];
                part[0] += (double)p[s] * (double)Ap[s];
            }
            group_sum<1>(part, red);
            const int c = c0 + g + groups * q;
            if (lt == 0 && have[q]) bufA[c] = part[0];
        }
        if (!grid_barrier(bar, epoch, ws.err, gridDim.x)) goto finish;
        {
            double tot[1];
            const int comp[1] = {0};
            scene_sums<1>(bufA, cb, ce, comp, tot, red, ws.tiles);
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
            for (int m = 0; m < 4; ++m) {
                const int s = q * 4 + m;
                const Cell cl = tile_cell(my[q], n, lt, m);
                if (!have[q] || !cl.ok) continue;
                x[s] = __fadd_rn(x[s], __fmul_rn(alpha, p[s]));
                r[s] = __fsub_rn(r[s], __fmul_rn(alpha, Ap[s]));
                z[s] = __fmul_rn(D[s], r[s]);
                zg[cl.t] = z[s];
                part[0] += (double)r[s] * (double)r[s];
                part[1] += (double)r[s] * (double)z[s];
            }
            group_sum<2>(part, red);
            const int c = c0 + g + groups * q;
            if (lt == 0 && have[q]) {
                bufB[1 * ws.tiles + c] = part[0];
                bufB[2 * ws.tiles + c] = part[1];
            }
        }
        if (!grid_barrier(bar, epoch, ws.err, gridDim.x)) goto finish;
        {
            double tot[2];
            const int comp[2] = {1, 2};
            scene_sums<2>(bufB, cb, ce, comp, tot, red, ws.tiles);
            if (threadIdx.x == 0) update_scalars(Ls, HEAT, tot[0], tot[1], kit);
            __syncthreads();
        }
    }
    // ------------------------------------------------------------------ write the solution back
#pragma unroll
    for (int q = 0; q < MAXC; ++q) {
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const Cell cl = tile_cell(my[q], n, lt, m);
            if (have[q] && cl.ok) xg[cl.t] = x[q * 4 + m];
        }
    }
    if (!HEAT) {
        // grid.py:140-153: the projection reads p at neighbour cells owned by other blocks
        if (!grid_barrier(bar, epoch, ws.err, gridDim.x)) goto finish;
        const float dtr = (float)(dt_d / S.rho);
#pragma unroll
        for (int q = 0; q < MAXC; ++q) {
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const Cell cl = tile_cell(my[q], n, lt, m);
                if (have[q] && cl.ok)
                    project_cell(S, S.u[par ^ 1], S.v[par ^ 1], S.w[par ^ 1], S.p, x[q * 4 + m], dtr, h, cl);
            }
        }
    }
finish:
    if (TMA && *(volatile int*)ws.err) {
        // leave no copy in flight: a timed-out wait is retried (bounded) before the block exits
#pragma unroll
        for (int q = 0; q < MAXC; ++q)
            if (have[q]) mbar_wait(&mbar[g * MAXC + q], phase_bit ^ 1u);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) write_stats(S, Ls, HEAT, *(volatile int*)ws.err != 0, par);
}

// ============================================================================= resident pressure CG with TMA staging
// Same mapping, arithmetic and reduction trees as k_pcg / k_pcg_res, with less state per thread: the search direction
// of the own cells is read from the staged box (its centre), A p is parked in the p_{k-1} box (dead once p_k is
// formed), so a thread keeps only x, r and D of its cells in registers.  One group reduction per phase covers all the
// thread's tiles.
// Set-up of one heat cell from the staged boxes (x0 with a one-cell halo at B, then the face-diffusivity boxes and the
// flag byte box at F): setup_cell<true>'s operations in its order on the same values (heat.py:198-203 with k_heat_diag
// and neighbour_terms, use_fixed = 0).  Box offsets as in the iterations' stencil.
__device__ __forceinline__ void heat_setup_box(const float* __restrict__ B, const float* __restrict__ F, float b, float c_dt,
                                               const Cell& cl, int n, int bi, int bj, int bk, float& bo, float& d,
                                               float& r, float& xo) {
    const float* axb = F;
    const float* ayb = axb + kBX;
    const float* azb = ayb + kBY;
    const unsigned char* flb = reinterpret_cast<const unsigned char*>(azb + kBW);
    const int o = (bi + 1) * 400 + (bj + 1) * 40 + (bk + 4);
    const int of = (bi + 1) * 640 + (bj + 1) * 64 + (bk + 16);
    const float xc = B[o];
    bo = b;
    xo = xc;
    if (flb[of] & 1) {
        d = 1.0f;
        r = __fsub_rn(b, xc);
        return;
    }
    const bool in[6] = {cl.i > 0, cl.i < n - 1, cl.j > 0, cl.j < n - 1, cl.k > 0, cl.k < n - 1};
    const float kf[6] = {axb[bi * 256 + bj * 32 + bk], axb[(bi + 1) * 256 + bj * 32 + bk], ayb[bi * 288 + bj * 32 + bk],
                         ayb[bi * 288 + (bj + 1) * 32 + bk], azb[bi * 288 + bj * 36 + bk], azb[bi * 288 + bj * 36 + bk + 1]};
    const int step[6] = {-400, 400, -40, 40, -1, 1}, fstep[6] = {-640, 640, -64, 64, -1, 1};
    float sd = 0.0f, nt = 0.0f;
#pragma unroll
    for (int s = 0; s < 6; ++s)
        if (in[s]) sd = __fadd_rn(sd, kf[s]);
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        if (!in[s]) continue;
        nt = __fadd_rn(nt, (flb[of + fstep[s]] & 1) ? __fmul_rn(kf[s], xc) : __fmul_rn(kf[s], __fsub_rn(xc, B[o + step[s]])));
    }
    d = __fdiv_rn(1.0f, __fadd_rn(1.0f, __fmul_rn(c_dt, sd)));
    r = __fsub_rn(b, __fadd_rn(xc, __fmul_rn(c_dt, nt)));
}

template <bool HEAT, int MAXC>
__global__ void __launch_bounds__(MAXC == 1 ? 1024 : (MAXC == 2 ? 768 : 512), 1)
    k_pcg_tma(const hf_scene* __restrict__ scenes, const TileItem* __restrict__ tiles, int tile_lo, int tile_hi,
              double dt_d, Workspace ws, const __grid_constant__ TileMaps maps) {
    constexpr int CPT = 4 * MAXC;
    constexpr int SLOT = HEAT ? kHeatSlotFloats : kSlotFloats;
    extern __shared__ __align__(128) float sm_raw[];
    float* sm_boxes = align128_shared(sm_raw);
    __shared__ double red[kRedComps * 32];
    __shared__ LocalScene Ls;
    __shared__ __align__(8) unsigned long long mbar[4 * 3];
    __shared__ TileItem my_s[4 * 3];
    const int groups = blockDim.x >> 8, g = threadIdx.x >> 8, lt = threadIdx.x & 255;
    const int c0 = tile_lo + (int)(((long long)(tile_hi - tile_lo) * blockIdx.x) / gridDim.x);
    const int c1 = tile_lo + (int)(((long long)(tile_hi - tile_lo) * (blockIdx.x + 1)) / gridDim.x);
    const int sidx = tiles[c0].scene;
    const hf_scene& S = scenes[sidx];
    const int n = S.n, N = n * n * n;
    const int par = S.state->parity;
    unsigned* bar = ws.bar + (HEAT ? 0 : kMaxLanes);
    unsigned epoch = 0;
    const float h = (float)S.h, hh = __fmul_rn(h, h), c_dt = __fdiv_rn((float)dt_d, hh);
    const DivBy hhd = div_by(hh);
    double* bufA = ws.partA;
    double* bufB = ws.partB;
    const int cb = ws.tile_begin[sidx], ce = ws.tile_begin[sidx + 1];
    float* xg = HEAT ? S.T[par ^ 1] : S.p;
    float* zg = S.cg_z;
    // the group's tiles in shared memory (registers held through the solve make the stencil phases spill)
    TileItem* const my = my_s + g * MAXC;
    bool have[MAXC];
#pragma unroll
    for (int q = 0; q < MAXC; ++q) have[q] = c0 + g + groups * q < c1;
    if (lt < MAXC) {
        const int c = c0 + g + groups * lt;
        my[lt] = tiles[c < c1 ? c : c0];
    }
    unsigned phase_bit = 0;
    // the z and p_{k-1} boxes of iteration kit, requested by thread lt == 0 of each group; the next iteration's are
    // requested right after the barrier that ends phase B, before the scene sums, so the copy overlaps them
    auto issue_boxes = [&](int kit) {
        if (lt != 0) return;
        asm volatile("fence.proxy.async.global;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
#pragma unroll
        for (int q = 0; q < MAXC; ++q) {
            if (!have[q]) continue;
            float* slot = sm_boxes + (size_t)(g * MAXC + q) * SLOT;
            unsigned long long* mb = &mbar[g * MAXC + q];
            mbar_expect_tx(mb, (unsigned)((kit == 1 ? 1 : 2) * kBZ * sizeof(float)));
            tma_load_3d(slot, &maps.z, my[q].k0 - 4, my[q].j0 - 1, my[q].i0 - 1, mb);
            if (kit != 1)
                tma_load_3d(slot + kBZ, ((kit - 1) & 1) ? &maps.p1 : &maps.p0, my[q].k0 - 4, my[q].j0 - 1, my[q].i0 - 1,
                            mb);
        }
    };
    bool requested = false;   // the next iteration's boxes are in flight
    if (lt == 0) {
#pragma unroll
        for (int q = 0; q < MAXC; ++q) mbar_init(&mbar[g * MAXC + q], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    float x[CPT], r[CPT], D[CPT];
    // heat: x0 (the advected T, into the z slot), the face diffusivities and the cell flags with halo are staged by
    // TMA before the set-up, which then reads them from shared memory; the coefficient boxes stay for the whole solve
    if (HEAT) {
        if (lt == 0) {
            asm volatile("fence.proxy.async.global;" ::: "memory");
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
#pragma unroll
            for (int q = 0; q < MAXC; ++q) {
                if (!have[q]) continue;
                float* slot = sm_boxes + (size_t)(g * MAXC + q) * SLOT;
                unsigned long long* mb = &mbar[g * MAXC + q];
                mbar_expect_tx(mb, (unsigned)((kBZ + kBX + kBY + kBW) * sizeof(float) + kBF));
                tma_load_3d(slot, (par ^ 1) ? &maps.t1 : &maps.t0, my[q].k0 - 4, my[q].j0 - 1, my[q].i0 - 1, mb);
                tma_load_3d(slot + 2 * kBZ, &maps.hkx, my[q].k0, my[q].j0, my[q].i0, mb);
                tma_load_3d(slot + 2 * kBZ + kBX, &maps.hky, my[q].k0, my[q].j0, my[q].i0, mb);
                tma_load_3d(slot + 2 * kBZ + kBX + kBY, &maps.hkzc, my[q].k0, my[q].j0, my[q].i0, mb);
                tma_load_3d(slot + 2 * kBZ + kBX + kBY + kBW, &maps.flags, my[q].k0 - 16, my[q].j0 - 1, my[q].i0 - 1, mb);
            }
        }
        bool ok = true;
#pragma unroll
        for (int q = 0; q < MAXC; ++q)
            if (have[q]) ok = mbar_wait(&mbar[g * MAXC + q], phase_bit) && ok;
        if (!ok) atomicExch(ws.err, 1);
        phase_bit ^= 1u;
    }
    // ------------------------------------------------------------------------------------------ prologue
    float mean = 0.0f;
    if (!HEAT) {
        double mm[1];
        const int comp[1] = {0};
        scene_sums<1>(ws.mean_part, ws.chunk_begin[sidx], ws.chunk_begin[sidx + 1], comp, mm, red, 0);
        mean = __double2float_rn(mm[0] / ((double)n * n * n));
    }
    {
        double part[3 * MAXC];
#pragma unroll
        for (int q = 0; q < MAXC; ++q) {
            part[3 * q] = part[3 * q + 1] = part[3 * q + 2] = 0.0;
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const int s = q * 4 + m;
                x[s] = r[s] = D[s] = 0.0f;
                const Cell cl = tile_cell(my[q], n, lt, m);
                if (!have[q] || !cl.ok) continue;
                float b, d, rr, xc;
                if (HEAT) {
                    const float* slot = sm_boxes + (size_t)(g * MAXC + q) * SLOT;
                    heat_setup_box(slot, slot + 2 * kBZ, S.hrhs[cl.t], c_dt, cl, n, m, lt >> 5, lt & 31, b, d, rr, xc);
                } else {
                    setup_cell<HEAT>(S, xg, mean, hh, c_dt, cl, b, d, rr);
                    xc = xg[cl.t];
                }
                const float z = __fmul_rn(d, rr);
                x[s] = xc;
                D[s] = d;
                r[s] = rr;
                zg[cl.t] = z;
                part[3 * q] += (double)b * (double)b;
                part[3 * q + 1] += (double)rr * (double)rr;
                part[3 * q + 2] += (double)rr * (double)z;
            }
        }
        group_sum<3 * MAXC>(part, red);
#pragma unroll
        for (int q = 0; q < MAXC; ++q) {
            const int c = c0 + g + groups * q;
            if (lt == 0 && have[q]) {
                bufB[c] = part[3 * q];
                bufB[1 * ws.tiles + c] = part[3 * q + 1];
                bufB[2 * ws.tiles + c] = part[3 * q + 2];
            }
        }
    }
    // the tiles' face fractions stay in shared memory for the whole solve (heat: staged before the set-up)
    if (!HEAT && lt == 0) {
#pragma unroll
        for (int q = 0; q < MAXC; ++q) {
            if (!have[q]) continue;
            float* slot = sm_boxes + (size_t)(g * MAXC + q) * SLOT;
            unsigned long long* mb = &mbar[g * MAXC + q];
            mbar_expect_tx(mb, (unsigned)((kBX + kBY + kBW) * sizeof(float)));
            tma_load_3d(slot + 2 * kBZ, &maps.ax, my[q].k0, my[q].j0, my[q].i0, mb);
            tma_load_3d(slot + 2 * kBZ + kBX, &maps.ayc, my[q].k0, my[q].j0, my[q].i0, mb);
            tma_load_3d(slot + 2 * kBZ + kBX + kBY, &maps.azc, my[q].k0, my[q].j0, my[q].i0, mb);
        }
    }
    if (!HEAT) {
        bool ok = true;
#pragma unroll
        for (int q = 0; q < MAXC; ++q)
            if (have[q]) ok = mbar_wait(&mbar[g * MAXC + q], phase_bit) && ok;
        if (!ok) atomicExch(ws.err, 1);
        phase_bit ^= 1u;
    }
    if (!grid_barrier(bar, epoch, ws.err, gridDim.x)) goto finish;
    issue_boxes(1);
    requested = true;
    {
        double tot[3];
        const int comp[3] = {0, 1, 2};
        scene_sums<3>(bufB, cb, ce, comp, tot, red, ws.tiles);
        if (threadIdx.x == 0) {
            init_scalars(Ls, S, HEAT, tot, N);
            Ls.mean = (double)mean;
        }
        __syncthreads();
    }
    // ------------------------------------------------------------------------------------------ iterations
    for (int kit = 1; Ls.live; ++kit) {
        const float beta = Ls.beta;
        const bool first = kit == 1;
        float* pnew = S.cg_p[kit & 1];
        // phase A: stage z and p_{k-1} with halo (requested after the previous barrier), form p_k in place, Ap from
        // shared memory
        if (!requested) issue_boxes(kit);
        requested = false;
        {
            bool ok = true;
#pragma unroll
            for (int q = 0; q < MAXC; ++q)
                if (have[q]) ok = mbar_wait(&mbar[g * MAXC + q], phase_bit) && ok;
            if (!ok) atomicExch(ws.err, 1);
            phase_bit ^= 1u;
        }
        if (!first) {
#pragma unroll
            for (int q = 0; q < MAXC; ++q) {
                if (!have[q]) continue;
                float* slot = sm_boxes + (size_t)(g * MAXC + q) * SLOT;
                for (int e = lt; e < kBZ; e += 256) slot[e] = __fadd_rn(slot[e], __fmul_rn(beta, slot[kBZ + e]));
            }
        }
        asm volatile("bar.sync %0, 256;" ::"r"(g + 1) : "memory");
        {
            double part[MAXC];
#pragma unroll
            for (int q = 0; q < MAXC; ++q) {
                part[q] = 0.0;
                float* slot = sm_boxes + (size_t)(g * MAXC + q) * SLOT;
                const float* Pb = slot;
                float* Apb = slot + kBZ;   // the p_{k-1} box is dead now: A p goes to its centre
                const float* axb = slot + 2 * kBZ;
                const float* ayb = axb + kBX;
                const float* azb = ayb + kBY;
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                    const Cell cl = tile_cell(my[q], n, lt, m);
                    if (!have[q] || !cl.ok) continue;
                    const int bi = m, bj = lt >> 5, bk = lt & 31;
                    const int o = (bi + 1) * 400 + (bj + 1) * 40 + (bk + 4);
                    const float pc = Pb[o];
                    float ap;
                    if (HEAT) {
                        // heat.py:94-105 with heat.py:55-91 neighbour_terms (use_fixed = 0): identity rows on fixed
                        // cells, fixed neighbours enter as kappa_f x_c
                        const unsigned char* flb = reinterpret_cast<const unsigned char*>(azb + kBW);
                        const int of = (bi + 1) * 640 + (bj + 1) * 64 + (bk + 16);
                        if (flb[of] & 1) {
                            ap = pc;
                        } else {
                            float acc = 0.0f;
                            float kf;
                            if (cl.i > 0) {
                                kf = axb[bi * 256 + bj * 32 + bk];
                                acc = __fadd_rn(acc, (flb[of - 640] & 1) ? __fmul_rn(kf, pc) : __fmul_rn(kf, __fsub_rn(pc, Pb[o - 400])));
                            }
                            if (cl.i < n - 1) {
                                kf = axb[(bi + 1) * 256 + bj * 32 + bk];
                                acc = __fadd_rn(acc, (flb[of + 640] & 1) ? __fmul_rn(kf, pc) : __fmul_rn(kf, __fsub_rn(pc, Pb[o + 400])));
                            }
                            if (cl.j > 0) {
                                kf = ayb[bi * 288 + bj * 32 + bk];
                                acc = __fadd_rn(acc, (flb[of - 64] & 1) ? __fmul_rn(kf, pc) : __fmul_rn(kf, __fsub_rn(pc, Pb[o - 40])));
                            }
                            if (cl.j < n - 1) {
                                kf = ayb[bi * 288 + (bj + 1) * 32 + bk];
                                acc = __fadd_rn(acc, (flb[of + 64] & 1) ? __fmul_rn(kf, pc) : __fmul_rn(kf, __fsub_rn(pc, Pb[o + 40])));
                            }
                            if (cl.k > 0) {
                                kf = azb[bi * 288 + bj * 36 + bk];
                                acc = __fadd_rn(acc, (flb[of - 1] & 1) ? __fmul_rn(kf, pc) : __fmul_rn(kf, __fsub_rn(pc, Pb[o - 1])));
                            }
                            if (cl.k < n - 1) {
                                kf = azb[bi * 288 + bj * 36 + bk + 1];
                                acc = __fadd_rn(acc, (flb[of + 1] & 1) ? __fmul_rn(kf, pc) : __fmul_rn(kf, __fsub_rn(pc, Pb[o + 1])));
                            }
                            ap = __fadd_rn(pc, __fmul_rn(c_dt, acc));
                        }
                    } else {
                        float acc = 0.0f;
                        if (cl.i > 0) acc = __fadd_rn(acc, __fmul_rn(axb[bi * 256 + bj * 32 + bk], __fsub_rn(pc, Pb[o - 400])));
                        if (cl.i < n - 1)
                            acc = __fadd_rn(acc, __fmul_rn(axb[(bi + 1) * 256 + bj * 32 + bk], __fsub_rn(pc, Pb[o + 400])));
                        if (cl.j > 0) acc = __fadd_rn(acc, __fmul_rn(ayb[bi * 288 + bj * 32 + bk], __fsub_rn(pc, Pb[o - 40])));
                        if (cl.j < n - 1)
                            acc = __fadd_rn(acc, __fmul_rn(ayb[bi * 288 + (bj + 1) * 32 + bk], __fsub_rn(pc, Pb[o + 40])));
                        if (cl.k > 0) acc = __fadd_rn(acc, __fmul_rn(azb[bi * 288 + bj * 36 + bk], __fsub_rn(pc, Pb[o - 1])));
                        if (cl.k < n - 1)
                            acc = __fadd_rn(acc, __fmul_rn(azb[bi * 288 + bj * 36 + bk + 1], __fsub_rn(pc, Pb[o + 1])));
                        ap = div_rn(acc, hhd);
                    }
                    Apb[o] = ap;
                    pnew[cl.t] = pc;
                    part[q] += (double)pc * (double)ap;
                }
            }
            group_sum<MAXC>(part, red);
#pragma unroll
            for (int q = 0; q < MAXC; ++q) {
                const int c = c0 + g + groups * q;
                if (lt == 0 && have[q]) bufA[c] = part[q];
            }
        }
        if (!grid_barrier(bar, epoch, ws.err, gridDim.x)) goto finish;
        {
            double tot[1];
            const int comp[1] = {0};
            scene_sums<1>(bufA, cb, ce, comp, tot, red, ws.tiles);
            if (threadIdx.x == 0) {
                Ls.pAp = tot[0];
                Ls.alpha = __double2float_rn(Ls.rz / tot[0]);
            }
            __syncthreads();
        }
        // phase B: x += alpha p, r -= alpha Ap, z = D r; publish z; r.r and r.z
        {
            const float alpha = Ls.alpha;
            double part[2 * MAXC];
#pragma unroll
            for (int q = 0; q < MAXC; ++q) {
                part[2 * q] = part[2 * q + 1] = 0.0;
                const float* slot = sm_boxes + (size_t)(g * MAXC + q) * SLOT;
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                    const int s = q * 4 + m;
                    const Cell cl = tile_cell(my[q], n, lt, m);
                    if (!have[q] || !cl.ok) continue;
                    const int o = (m + 1) * 400 + ((lt >> 5) + 1) * 40 + ((lt & 31) + 4);
                    x[s] = __fadd_rn(x[s], __fmul_rn(alpha, slot[o]));
                    r[s] = __fsub_rn(r[s], __fmul_rn(alpha, slot[kBZ + o]));
                    const float z = __fmul_rn(D[s], r[s]);
                    zg[cl.t] = z;
                    part[2 * q] += (double)r[s] * (double)r[s];
                    part[2 * q + 1] += (double)r[s] * (double)z;
                }
            }
            group_sum<2 * MAXC>(part, red);
#pragma unroll
            for (int q = 0; q < MAXC; ++q) {
                const int c = c0 + g + groups * q;
                if (lt == 0 && have[q]) {
                    bufB[1 * ws.tiles + c] = part[2 * q];
                    bufB[2 * ws.tiles + c] = part[2 * q + 1];
                }
            }
        }
        if (!grid_barrier(bar, epoch, ws.err, gridDim.x)) goto finish;
        issue_boxes(kit + 1);
        requested = true;
        {
            double tot[2];
            const int comp[2] = {1, 2};
            scene_sums<2>(bufB, cb, ce, comp, tot, red, ws.tiles);
            if (threadIdx.x == 0) update_scalars(Ls, HEAT, tot[0], tot[1], kit);
            __syncthreads();
        }
    }
    if (requested) {
        // the solve ended: the boxes requested for an iteration that does not run are waited for (no copy in flight)
        bool ok = true;
#pragma unroll
        for (int q = 0; q < MAXC; ++q)
            if (have[q]) ok = mbar_wait(&mbar[g * MAXC + q], phase_bit) && ok;
        if (!ok) atomicExch(ws.err, 1);
        phase_bit ^= 1u;
        requested = false;
    }
    // -------------------------------------------------- write x back, then (pressure) project the faces
#pragma unroll
    for (int q = 0; q < MAXC; ++q) {
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const Cell cl = tile_cell(my[q], n, lt, m);
            if (have[q] && cl.ok) xg[cl.t] = x[q * 4 + m];
        }
    }
    if (!HEAT) {
        if (!grid_barrier(bar, epoch, ws.err, gridDim.x)) goto finish;
        const float dtr = (float)(dt_d / S.rho);
#pragma unroll
        for (int q = 0; q < MAXC; ++q) {
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const Cell cl = tile_cell(my[q], n, lt, m);
                if (have[q] && cl.ok)
                    project_cell(S, S.u[par ^ 1], S.v[par ^ 1], S.w[par ^ 1], S.p, x[q * 4 + m], dtr, h, cl);
            }
        }
    }
finish:
    if (*(volatile int*)ws.err) {
        // leave no copy in flight: a timed-out wait is retried (bounded) before the block exits
#pragma unroll
        for (int q = 0; q < MAXC; ++q)
            if (have[q]) mbar_wait(&mbar[g * MAXC + q], phase_bit ^ 1u);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) write_stats(S, Ls, HEAT, *(volatile int*)ws.err != 0, par);
}

// ===================================================== resident pressure CG, one reduction point per iteration
// Jacobi-PCG of the pressure system of one scene (n % 4 == 0) with ONE grid barrier per iteration instead of two.  The
// vectors follow the classic recurrences (A p formed from p every iteration, r -= alpha A p, p = z + beta p with
// z ~ D r); only beta is obtained differently.  In iteration k every block forms, next to p_k . A p_k, the direct
// r_k . r_k and r_k . z_k of its cells and the two terms A p_k . z_k and A p_k . D A p_k, so that one scene sum gives
//     alpha_k = rz_k / pAp_k,   rz_{k+1} = rz_k - 2 alpha_k (A p_k . z_k) + alpha_k^2 (A p_k . D A p_k),
//     beta_{k+1} = rz_{k+1} / rz_k
// (the expansion of (r_k - alpha A p_k) . D (r_k - alpha A p_k) used by D'Azevedo, Eijkhout & Romine, "Conjugate
// gradient algorithms with reduced synchronization overhead on distributed memory multiprocessors", 1993).  rz_k is
// the direct sum of every iteration, so the expansion never accumulates; it differs from the direct rz_{k+1} only by
// the binary32 rounding of r_{k+1} (~1e-7 relative), so beta moves by that much and the solve converges like the
// classic one (the same iteration counts and x within ~1e-8 relative on the benchmark scene's systems; at tolerance
// 1e-6 too).  The convergence test is the classic one on the direct r_k . r_k, taken at the barrier after r_k was
// formed: a solve stops with the same x and reports the same iteration count.
//
// Partials: a thread adds the five products of its cells in cell order, the warp butterfly and the group's 8 warps in
// order give one set per 256-thread group, and every block sums the groups' sets in group order (the set-up's three
// sums stay per tile).  The tree is fixed for a given grid, so a solve is deterministic; unlike the classic variants'
// per-tile tree it depends on the launch shape (this kernel only runs single-scene plans).
//
// Halo: iteration k + 1 needs p_{k+1} = z_{k+1} + beta p_k at the tile's face neighbours, which belong to other
// blocks.  Every block publishes, for the cells on its tiles' faces, z_k' = D r_k and q_k = D A p_k (double-buffered:
// z' in cg_r / cg_z, q in cg_Ap / hdiag -- the heat diagonal is dead while the pressure system is solved).  Right
// after the barrier a block requests the z', q values of its tiles' 832 face-neighbour points (cp.async), in flight
// while it sums the partials; then every p_{k+1} in its boxes, own cells and neighbours alike, is formed by the same
// operations from the same values, z = z' - alpha q, p = z + beta p, so all blocks agree bit for bit and no block
// needs another's p: the p boxes (one-cell halo) are loaded once, from the published p0 (TMA), and advanced in place.
// State: r, A p and D of a thread's cells in registers; x, the p box, the face-fraction boxes (TMA, once) and the
// halo staging in shared memory.
constexpr int kOneFaces = kBZ;                            // slot offset of the face-fraction boxes
constexpr int kOneCells = kBZ + kBX + kBY + kBW;          // slot offset of x (1024 floats)
constexpr int kOneHalo = kOneCells + 1024;                // slot offset of the halo staging: z' and q of 832 points
constexpr int kOneHaloPts = 832;
constexpr int kOneSlotFloats = kOneHalo + 2 * kOneHaloPts;   // 8672 floats = 34,688 bytes (a multiple of 128)
constexpr int kOneComps = 5;                              // partials per group: pAp, rr, rz, Ap.z, Ap.D.Ap
static_assert(kOneSlotFloats % 32 == 0, "slots stay 128-byte aligned");

// grid.py:94-115 k_laplacian of one tile cell from a staged box (centre offset o) and the tile's face boxes
__device__ __forceinline__ float lap_box(const float* __restrict__ B, const float* __restrict__ axb,
                                         const float* __restrict__ ayb, const float* __restrict__ azb, const Cell& cl,
                                         int n, int bi, int bj, int bk, int o, const DivBy& hh) {
    const float pc = B[o];
    float acc = 0.0f;
    if (cl.i > 0) acc = __fadd_rn(acc, __fmul_rn(axb[bi * 256 + bj * 32 + bk], __fsub_rn(pc, B[o - 400])));
    if (cl.i < n - 1) acc = __fadd_rn(acc, __fmul_rn(axb[(bi + 1) * 256 + bj * 32 + bk], __fsub_rn(pc, B[o + 400])));
    if (cl.j > 0) acc = __fadd_rn(acc, __fmul_rn(ayb[bi * 288 + bj * 32 + bk], __fsub_rn(pc, B[o - 40])));
    if (cl.j < n - 1) acc = __fadd_rn(acc, __fmul_rn(ayb[bi * 288 + (bj + 1) * 32 + bk], __fsub_rn(pc, B[o + 40])));
    if (cl.k > 0) acc = __fadd_rn(acc, __fmul_rn(azb[bi * 288 + bj * 36 + bk], __fsub_rn(pc, B[o - 1])));
    if (cl.k < n - 1) acc = __fadd_rn(acc, __fmul_rn(azb[bi * 288 + bj * 36 + bk + 1], __fsub_rn(pc, B[o + 1])));
    return div_rn(acc, hh);
}

// Face-neighbour point u (0..3) of thread lt around a 4 x 8 x 32 tile, as box offsets (bi, bj, bk in -1..4, -1..8,
// -1..32): the two i faces (256 points each), the two j faces (128 each) and the two k faces (32 each) -- 832 points,
// three or four per thread, consecutive threads on consecutive k; staging index u * 256 + lt.  False when the thread
// has no point u.
__device__ __forceinline__ bool halo_point(int lt, int u, int& bi, int& bj, int& bk) {
    if (u == 0 || u == 1) {
        bi = u == 0 ? -1 : 4;
        bj = lt >> 5;
        bk = lt & 31;
        return true;
    }
    if (u == 2) {
        bi = (lt & 127) >> 5;
        bj = lt < 128 ? -1 : 8;
        bk = lt & 31;
        return true;
    }
    if (lt >= 64) return false;
    bi = (lt & 31) >> 3;
    bj = lt & 7;
    bk = lt < 32 ? -1 : 32;
    return true;
}

// global cell of face-neighbour point u of thread lt around tile ti, or -1 (no point, or outside the domain)
__device__ __forceinline__ int halo_cell(const TileItem& ti, int n, int lt, int u) {
    int bi = 0, bj = 0, bk = 0;
    if (!halo_point(lt, u, bi, bj, bk)) return -1;
    const int gi = ti.i0 + bi, gj = ti.j0 + bj, gk = ti.k0 + bk;
    if (gi < 0 || gi >= n || gj < 0 || gj >= n || gk < 0 || gk >= n) return -1;
    return (gi * n + gj) * n + gk;
}

__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}

template <int MAXC>
__global__ void __launch_bounds__(MAXC == 1 ? 1024 : (MAXC == 2 ? 768 : 512), 1)
    k_pcg_one(const hf_scene* __restrict__ scenes, const TileItem* __restrict__ tiles, int tile_lo, int tile_hi,
              double dt_d, Workspace ws, const __grid_constant__ TileMaps maps) {
    constexpr int CPT = 4 * MAXC;
    extern __shared__ __align__(128) float sm_raw[];
    float* sm_slots = align128_shared(sm_raw);
    __shared__ double red[kOneComps * 3 * 32];   // five partials per warp (the set-up: three of up to three tiles)
    __shared__ unsigned hmask_s[1024];
    __shared__ TileItem my_s[4 * 3];
    __shared__ LocalScene Ls;
    __shared__ __align__(8) unsigned long long mbar[4 * 3];
    const int groups = blockDim.x >> 8, g = threadIdx.x >> 8, lt = threadIdx.x & 255;
    const int c0 = tile_lo + (int)(((long long)(tile_hi - tile_lo) * blockIdx.x) / gridDim.x);
    const int c1 = tile_lo + (int)(((long long)(tile_hi - tile_lo) * (blockIdx.x + 1)) / gridDim.x);
    const int sidx = tiles[c0].scene;
    const hf_scene& S = scenes[sidx];
    const int n = S.n, N = n * n * n;
    const int par = S.state->parity;
    unsigned* bar = ws.bar + kMaxLanes;
    unsigned epoch = 0;
    const float h = (float)S.h, hh = __fmul_rn(h, h);
    const DivBy hhd = div_by(hh);
    double* const bufA = ws.partA;
    double* const bufB = ws.partB;
    const int cb = ws.tile_begin[sidx], ce = ws.tile_begin[sidx + 1];
    // the iterations' partials: one per 256-thread group, unit = block x groups + group (the launch keeps the units
    // within the tile count that the partial buffers are sized for)
    const int units = (int)gridDim.x * groups, unit = (int)blockIdx.x * groups + g;
    float* xg = S.p;
    // the group's tiles (shared memory, like the halo mask below: registers held through the solve make the stencil
    // phase spill)
    TileItem* const my = my_s + g * MAXC;
    bool have[MAXC];
#pragma unroll
    for (int q = 0; q < MAXC; ++q) have[q] = c0 + g + groups * q < c1;
    if (lt < MAXC) {
        const int c = c0 + g + groups * lt;
        my[lt] = tiles[c < c1 ? c : c0];
    }
    auto slot_of = [&](int q) { return sm_slots + (size_t)(g * MAXC + q) * kOneSlotFloats; };
    unsigned phase_bit = 0;
    auto wait_boxes = [&]() {
        bool ok = true;
#pragma unroll
        for (int q = 0; q < MAXC; ++q)
            if (have[q]) ok = mbar_wait(&mbar[g * MAXC + q], phase_bit) && ok;
        if (!ok) atomicExch(ws.err, 1);
        phase_bit ^= 1u;
    };
    if (lt == 0) {
#pragma unroll
        for (int q = 0; q < MAXC; ++q) mbar_init(&mbar[g * MAXC + q], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // bit 4 q + u of hmask_s[thread]: the thread's face-neighbour point u of tile q exists and lies in the domain
    {
        unsigned hm = 0;
#pragma unroll
        for (int q = 0; q < MAXC; ++q)
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (have[q] && halo_cell(my[q], n, lt, u) >= 0) hm |= 1u << (4 * q + u);
        hmask_s[threadIdx.x] = hm;
    }
    float r[CPT], ap[CPT], dg[CPT];
    int k = 0;
    // ------------------------------------------------------------------------------------------ set-up
    float mean = 0.0f;
    {
        double mm[1];
        const int comp[1] = {0};
        scene_sums<1>(ws.mean_part, ws.chunk_begin[sidx], ws.chunk_begin[sidx + 1], comp, mm, red, 0);
        mean = __double2float_rn(mm[0] / ((double)n * n * n));
    }
    {
        // r0 = b - A x0, p0 = z0 = D r0 (published for the halo of A p0); partials b.b, r.r, r.z
        __syncthreads();   // red is free (the rhs mean above read it)
#pragma unroll
        for (int q = 0; q < MAXC; ++q) {
            double part[3] = {0.0, 0.0, 0.0};
            float* X = slot_of(q) + kOneCells;
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const int s = q * 4 + m, e = m * 256 + lt;
                r[s] = ap[s] = dg[s] = 0.0f;
                X[e] = 0.0f;
                const Cell cl = tile_cell(my[q], n, lt, m);
                if (!have[q] || !cl.ok) continue;
                float b, d, rr;
                setup_cell<false>(S, xg, mean, hh, 0.0f, cl, b, d, rr);
                const float z = __fmul_rn(d, rr);
                X[e] = xg[cl.t];
                dg[s] = d;
                r[s] = rr;
                S.cg_p[0][cl.t] = z;
                part[0] += (double)b * (double)b;
                part[1] += (double)rr * (double)rr;
                part[2] += (double)rr * (double)z;
            }
            stash_warp<3>(part, red, 3 * q);
        }
        publish_group<MAXC>(red, bufB, c0 + g, groups, c1, ws.tiles);
    }
    // the tiles' face fractions stay in shared memory for the whole solve
    if (lt == 0) {
#pragma unroll
        for (int q = 0; q < MAXC; ++q) {
            if (!have[q]) continue;
            float* slot = slot_of(q);
            unsigned long long* mb = &mbar[g * MAXC + q];
            mbar_expect_tx(mb, (unsigned)((kBX + kBY + kBW) * sizeof(float)));
            tma_load_3d(slot + kOneFaces, &maps.ax, my[q].k0, my[q].j0, my[q].i0, mb);
            tma_load_3d(slot + kOneFaces + kBX, &maps.ayc, my[q].k0, my[q].j0, my[q].i0, mb);
            tma_load_3d(slot + kOneFaces + kBX + kBY, &maps.azc, my[q].k0, my[q].j0, my[q].i0, mb);
        }
    }
    wait_boxes();
    if (!grid_barrier(bar, epoch, ws.err, gridDim.x)) goto finish;
    {
        double tot[3];
        const int comp[3] = {0, 1, 2};
        scene_sums<3>(bufB, cb, ce, comp, tot, red, ws.tiles);
        if (threadIdx.x == 0) {
            init_scalars(Ls, S, false, tot, N);
            Ls.mean = (double)mean;
        }
        __syncthreads();
    }
    if (!Ls.live) goto writeback;
    // ------------------------------------------------------------------------------------------ iterations
    // k = 0 forms A p0 from the published p0; k >= 1 first advances x, r and p with the scalars of iteration k - 1
    for (k = 0;; ++k) {
        const int prev = (k & 1) ^ 1;
        // k = 0: the p0 boxes (TMA), requested before the scene sums; after that the boxes stay in shared memory and
        // every block advances its own copy of p at its tiles' cells and face neighbours
        if (k == 0 && lt == 0) {
            asm volatile("fence.proxy.async.global;" ::: "memory");
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
#pragma unroll
            for (int q = 0; q < MAXC; ++q) {
                if (!have[q]) continue;
                unsigned long long* mb = &mbar[g * MAXC + q];
                mbar_expect_tx(mb, (unsigned)(kBZ * sizeof(float)));
                tma_load_3d(slot_of(q), &maps.p0, my[q].k0 - 4, my[q].j0 - 1, my[q].i0 - 1, mb);
            }
        }
        // k >= 1: the loads of this iteration's scene sums first, then the neighbours' z', q (cp.async), in flight
        // while the sums are formed
        double sv[kOneComps][2];
        if (k > 0) {
            if (groups >= 2)
                unit_loads<kOneComps, 2, 2>(prev ? bufB : bufA, units, sv);
            else
                unit_loads<kOneComps, 1, 2>(prev ? bufB : bufA, units, sv);
        }
        if (k > 0) {
            const float* Zp = prev ? S.cg_z : S.cg_r;
            const float* Qp = prev ? S.hdiag : S.cg_Ap;
            const unsigned hmask = hmask_s[threadIdx.x];
#pragma unroll
            for (int q = 0; q < MAXC; ++q) {
                float* stg = slot_of(q) + kOneHalo;
                const int tb = (my[q].i0 * n + my[q].j0) * n + my[q].k0;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    int bi = 0, bj = 0, bk = 0;
                    if (!((hmask >> (4 * q + u)) & 1u)) continue;
                    halo_point(lt, u, bi, bj, bk);
                    const int t = tb + (bi * n + bj) * n + bk;
                    cp_async4(stg + u * 256 + lt, Zp + t);
                    cp_async4(stg + kOneHaloPts + u * 256 + lt, Qp + t);
                }
            }
            asm volatile("cp.async.commit_group;" ::: "memory");
        }
        float alpha = 0.0f, beta = 0.0f;
        bool live = true;   // k = 0 runs only when the set-up left the scene live
        if (k > 0) {
            double tot[kOneComps];
            // pAp, rr, rz, Ap.z, Ap.D.Ap of iteration k - 1: the groups' partials in group order, in every thread
            if (groups >= 2)
                unit_sums<kOneComps, 2, 2>(prev ? bufB : bufA, units, sv, tot, red);
            else
                unit_sums<kOneComps, 1, 2>(prev ? bufB : bufA, units, sv, tot, red);
            // every thread derives the same test and scalars from the same sums (no broadcast through shared memory):
            // the classic test on r_{k-1} (formed in iteration k - 1); converged -> x_{k-1} is the solution
            const double pAp = tot[0], rr = tot[1], rz = tot[2];
            const bool above = rr > Ls.atol_sq;
            live = above && isfinite(rr) && (k - 1) < Ls.maxit;
            if (live) {
                const double a = rz / pAp;
                const double rz_next = rz - 2.0 * a * tot[3] + a * a * tot[4];
                alpha = __double2float_rn(a);
                beta = __double2float_rn(rz_next / rz);
            }
            if (threadIdx.x == 0) {
                Ls.iters = k - 1;
                Ls.rr = rr;
                Ls.rz = rz;
                Ls.pAp = pAp;
                if (!isfinite(rr)) Ls.status |= HF_SCENE_NONFINITE;
                if (!live && above && isfinite(rr)) Ls.status |= HF_SCENE_PRESSURE_MAXITER;
                Ls.live = live;
                Ls.alpha = alpha;
                Ls.beta = beta;
            }
        }
        if (k == 0) wait_boxes();
        if (k > 0) asm volatile("cp.async.wait_all;" ::: "memory");
        asm volatile("bar.sync %0, 256;" ::"r"(g + 1) : "memory");
        if (!live) break;
        if (k > 0) {
            // p_k everywhere in the boxes by one formula: z = z' - alpha q, p = z + beta p_{k-1}; own cells also
            // advance x and r
            const unsigned hmask = hmask_s[threadIdx.x];
#pragma unroll
            for (int q = 0; q < MAXC; ++q) {
                float* box = slot_of(q);
                const float* stg = box + kOneHalo;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    int bi = 0, bj = 0, bk = 0;
                    if (!((hmask >> (4 * q + u)) & 1u)) continue;
                    halo_point(lt, u, bi, bj, bk);
                    float& pb = box[(bi + 1) * 400 + (bj + 1) * 40 + (bk + 4)];
                    const float z = __fsub_rn(stg[u * 256 + lt], __fmul_rn(alpha, stg[kOneHaloPts + u * 256 + lt]));
                    pb = __fadd_rn(z, __fmul_rn(beta, pb));
                }
                float* X = box + kOneCells;
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                    const int s = q * 4 + m, e = m * 256 + lt;
                    const Cell cl = tile_cell(my[q], n, lt, m);
                    if (!have[q] || !cl.ok) continue;
                    float& pb = box[(m + 1) * 400 + ((lt >> 5) + 1) * 40 + ((lt & 31) + 4)];
                    const float zp = __fmul_rn(dg[s], r[s]), qv = __fmul_rn(dg[s], ap[s]);
                    const float z = __fsub_rn(zp, __fmul_rn(alpha, qv));
                    X[e] = __fadd_rn(X[e], __fmul_rn(alpha, pb));
                    r[s] = __fsub_rn(r[s], __fmul_rn(alpha, ap[s]));
                    pb = __fadd_rn(z, __fmul_rn(beta, pb));
                }
            }
            asm volatile("bar.sync %0, 256;" ::"r"(g + 1) : "memory");
        }
        // A p_k from the box; partials of iteration k; publish z_k' = D r_k and q_k = D A p_k
        {
            const int cur = k & 1;
            float* const Zc = cur ? S.cg_z : S.cg_r;
            float* const Qc = cur ? S.hdiag : S.cg_Ap;
            __syncthreads();   // red is free (the scene sums above read it)
            // the five partials of the thread's cells, in cell order (tile q, then m)
            double part[kOneComps] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int q = 0; q < MAXC; ++q) {
                const float* slot = slot_of(q);
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                    const int s = q * 4 + m;
                    const Cell cl = tile_cell(my[q], n, lt, m);
                    if (!have[q] || !cl.ok) continue;
                    const int bj = lt >> 5, bk = lt & 31, o = (m + 1) * 400 + (bj + 1) * 40 + (bk + 4);
                    const float pk = slot[o];
                    ap[s] = lap_box(slot, slot + kOneFaces, slot + kOneFaces + kBX, slot + kOneFaces + kBX + kBY, cl, n,
                                    m, bj, bk, o, hhd);
                    const float zp = __fmul_rn(dg[s], r[s]);
                    const double d = dg[s], a = ap[s], rs = r[s], z = zp;
                    part[0] += (double)pk * a;
                    part[1] += rs * rs;
                    part[2] += rs * z;
                    part[3] += a * z;
                    part[4] += a * (d * a);
                    // only cells on the tile's faces are another tile's face neighbours
                    if (m == 0 || m == 3 || bj == 0 || bj == 7 || bk == 0 || bk == 31) {
                        Zc[cl.t] = zp;
                        Qc[cl.t] = __fmul_rn(dg[s], ap[s]);
                    }
                }
            }
            stash_warp<kOneComps>(part, red, 0);
            publish_unit<kOneComps>(red, cur ? bufB : bufA, unit, units);
        }
        if (!grid_barrier(bar, epoch, ws.err, gridDim.x)) goto finish;
    }
writeback:
    // -------------------------------------------------- write x back, then project the faces
#pragma unroll
    for (int q = 0; q < MAXC; ++q) {
        const float* X = slot_of(q) + kOneCells;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const Cell cl = tile_cell(my[q], n, lt, m);
            if (have[q] && cl.ok) xg[cl.t] = X[m * 256 + lt];
        }
    }
    if (!grid_barrier(bar, epoch, ws.err, gridDim.x)) goto finish;
    {
        const float dtr = (float)(dt_d / S.rho);
#pragma unroll
        for (int q = 0; q < MAXC; ++q) {
            const float* X = slot_of(q) + kOneCells;
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const Cell cl = tile_cell(my[q], n, lt, m);
                if (have[q] && cl.ok)
                    project_cell(S, S.u[par ^ 1], S.v[par ^ 1], S.w[par ^ 1], S.p, X[m * 256 + lt], dtr, h, cl);
            }
        }
    }
finish:
    if (*(volatile int*)ws.err) {
        // leave no copy in flight: the last requested boxes are waited for again (bounded) before the block exits
#pragma unroll
        for (int q = 0; q < MAXC; ++q)
            if (have[q]) mbar_wait(&mbar[g * MAXC + q], phase_bit ^ 1u);
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    if (blockIdx.x == 0 && threadIdx.x == 0) write_stats(S, Ls, false, *(volatile int*)ws.err != 0, par);
}

const void* pcg_one_kernel(int maxc) {
    if (maxc == 1) return (const void*)k_pcg_one<1>;
    if (maxc == 2) return (const void*)k_pcg_one<2>;
    return (const void*)k_pcg_one<3>;
}

size_t pcg_one_smem(int groups, int maxc) { return (size_t)groups * maxc * kOneSlotFloats * sizeof(float) + 128; }

const void* pcg_kernel(bool heat, bool tma) {
    return heat ? (const void*)k_pcg<true, false> : tma ? (const void*)k_pcg<false, true> : (const void*)k_pcg<false, false>;
}

size_t pcg_stream_smem(bool tma) { return tma ? 2 * (size_t)kSlotFloats * sizeof(float) + 128 : 0; }

const void* pcg_resident_kernel(bool heat, int maxc, bool tma) {
    if (heat && tma) {
        if (maxc == 1) return (const void*)k_pcg_tma<true, 1>;
        if (maxc == 2) return (const void*)k_pcg_tma<true, 2>;
        return (const void*)k_pcg_tma<true, 3>;
    }
    if (heat) {
        if (maxc == 1) return (const void*)k_pcg_res<true, 1, false>;
        if (maxc == 2) return (const void*)k_pcg_res<true, 2, false>;
        return (const void*)k_pcg_res<true, 3, false>;
    }
    if (tma) {
        if (maxc == 1) return (const void*)k_pcg_tma<false, 1>;
        if (maxc == 2) return (const void*)k_pcg_tma<false, 2>;
        return (const void*)k_pcg_tma<false, 3>;
    }
    if (maxc == 1) return (const void*)k_pcg_res<false, 1, false>;
    if (maxc == 2) return (const void*)k_pcg_res<false, 2, false>;
    return (const void*)k_pcg_res<false, 3, false>;
}

int set_wait_limit(unsigned long long limit_ns, int absent_block) {
    if (cudaMemcpyToSymbol(c_wait_limit_ns, &limit_ns, sizeof limit_ns) != cudaSuccess) return HF_ERR_CUDA;
    if (cudaMemcpyToSymbol(c_absent_block, &absent_block, sizeof absent_block) != cudaSuccess) return HF_ERR_CUDA;
    return HF_OK;
}

size_t pcg_resident_smem(int groups, int maxc, bool tma, bool heat) {
    return tma ? (size_t)groups * maxc * (heat ? kHeatSlotFloats : kSlotFloats) * sizeof(float) + 128 : 0;
}

}  // namespace hf
