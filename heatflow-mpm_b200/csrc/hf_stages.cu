// hf_stages.cu -- the non-iterative stages of the air substep, batched over a scene table.
//
// The chunked kernels run one block per 1024-cell work item (scene, first cell): 256 threads taking the cells
// first + tid + 256*m, m = 0..3 (the divergence: 1024 threads, one cell each), so that warps read consecutive k (the
// contiguous axis) and every global access is coalesced.  The sampling stages run one 512-thread block per CG tile
// with the lattices around the tile staged in shared memory.  Face stages are organised by cell: a thread owns the
// three low faces u(i,j,k), v(i,j,k), w(i,j,k) of its cell and, on the last layer, the high wall face.
#include <climits>

#include "hf_device.cuh"
#include "hf_kernels.cuh"

namespace hf {

// ---------------------------------------------------------------------------------------------- index helpers
__device__ __forceinline__ int uidx(int n, int i, int j, int k) { return (i * n + j) * n + k; }            // (n+1,n,n)
__device__ __forceinline__ int vidx(int n, int i, int j, int k) { return (i * (n + 1) + j) * n + k; }      // (n,n+1,n)
__device__ __forceinline__ int widx(int n, int i, int j, int k) { return (i * n + j) * (n + 1) + k; }      // (n,n,n+1)

// ------------------------------------------------------------------------------------------------ particles
// solver.py:19-38 (k_scatter_particles) and heat.py:12-18 (k_scatter_heat): each weight is formed in binary32
// exactly as the reference's atomic operand, rounded to a 2^-40 fixed-point integer and added with an integer atomic,
// so the sum does not depend on the order in which particles arrive.
__device__ __forceinline__ void scatter_fx(long long* acc, float px, float py, float pz, float ox, float oy, float oz,
                                           float h, int nx, int ny, int nz, float val) {
    float gx = __fsub_rn(__fdiv_rn(px, h), ox);
    float gy = __fsub_rn(__fdiv_rn(py, h), oy);
    float gz = __fsub_rn(__fdiv_rn(pz, h), oz);
    int ix = (int)floorf(gx), iy = (int)floorf(gy), iz = (int)floorf(gz);
    float fx = __fsub_rn(gx, (float)ix), fy = __fsub_rn(gy, (float)iy), fz = __fsub_rn(gz, (float)iz);
#pragma unroll
    for (int dx = 0; dx < 2; ++dx) {
        int cx = clampi(ix + dx, 0, nx - 1);
        float wx = dx ? fx : __fsub_rn(1.0f, fx);
#pragma unroll
        for (int dy = 0; dy < 2; ++dy) {
            int cy = clampi(iy + dy, 0, ny - 1);
            float wy = dy ? fy : __fsub_rn(1.0f, fy);
#pragma unroll
            for (int dz = 0; dz < 2; ++dz) {
                int cz = clampi(iz + dz, 0, nz - 1);
                float wz = dz ? fz : __fsub_rn(1.0f, fz);
                float c = __fmul_rn(__fmul_rn(__fmul_rn(wx, wy), wz), val);
                long long q = __double2ll_rn((double)c * kFxScale);
                if (q) atomicAdd(reinterpret_cast<unsigned long long*>(acc + (cx * ny + cy) * nz + cz),
                                 static_cast<unsigned long long>(q));
            }
        }
    }
}

// Cells whose obstacle fields a particle can touch: floor(x/h) - 1 .. floor(x/h) + 1 per axis covers the cell lattice
// (offset 1/2) and the face lattices (offset 0 or 1/2), the high wall face included (it belongs to cell n-1).
__device__ __forceinline__ void footprint(float x, float h, int n, int& lo, int& hi) {
    const int c = (int)floorf(__fdiv_rn(x, h));
    lo = clampi(c - 1, 0, n - 1);
    hi = clampi(c + 1, 0, n - 1);
}

// One launch per substep for the particles' two passes: the footprint box of this substep (the cells whose obstacle
// fields a particle can touch, a min/max over particles) and the fixed-point scatter of solver.py:19-38 / heat.py:12-18.
__global__ void __launch_bounds__(kThreads) k_scatter(const hf_scene* __restrict__ scenes, int s) {
    const hf_scene& S = scenes[s];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = S.n;
    const float h = (float)S.h;
    {
        int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
        if (t < S.n_particles) {
#pragma unroll
            for (int d = 0; d < 3; ++d) footprint(S.pos[3 * t + d], h, n, lo[d], hi[d]);
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            lo[d] = __reduce_min_sync(0xffffffffu, lo[d]);
            hi[d] = __reduce_max_sync(0xffffffffu, hi[d]);
        }
        if ((threadIdx.x & 31) == 0 && lo[0] <= hi[0]) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                atomicMin(&S.state->box[d], lo[d]);
                atomicMax(&S.state->box[3 + d], hi[d]);
            }
        }
    }
    if (t >= S.n_particles) return;
    const float vol = (float)S.vol, k0 = (float)S.k_particle;
    const long long M = (long long)(n + 1) * (n + 1) * (n + 1);
    long long* acc = S.acc;
    const float px = S.pos[3 * t], py = S.pos[3 * t + 1], pz = S.pos[3 * t + 2];
    const float vx = S.pvel[3 * t], vy = S.pvel[3 * t + 1], vz = S.pvel[3 * t + 2];
    const float frac = __fdiv_rn(vol, __fmul_rn(__fmul_rn(h, h), h));
    scatter_fx(acc + 0 * M, px, py, pz, 0.5f, 0.5f, 0.5f, h, n, n, n, frac);
    scatter_fx(acc + 1 * M, px, py, pz, 0.0f, 0.5f, 0.5f, h, n + 1, n, n, __fmul_rn(frac, vx));
    scatter_fx(acc + 2 * M, px, py, pz, 0.5f, 0.0f, 0.5f, h, n, n + 1, n, __fmul_rn(frac, vy));
    scatter_fx(acc + 3 * M, px, py, pz, 0.5f, 0.5f, 0.0f, h, n, n, n + 1, __fmul_rn(frac, vz));
    scatter_fx(acc + 4 * M, px, py, pz, 0.0f, 0.5f, 0.5f, h, n + 1, n, n, k0);
    scatter_fx(acc + 5 * M, px, py, pz, 0.5f, 0.0f, 0.5f, h, n, n + 1, n, k0);
    scatter_fx(acc + 6 * M, px, py, pz, 0.5f, 0.5f, 0.0f, h, n, n, n + 1, k0);
    scatter_fx(acc + 7 * M, px, py, pz, 0.0f, 0.5f, 0.5f, h, n + 1, n, n, __fmul_rn(k0, vx));
    scatter_fx(acc + 8 * M, px, py, pz, 0.5f, 0.0f, 0.5f, h, n, n + 1, n, __fmul_rn(k0, vy));
    scatter_fx(acc + 9 * M, px, py, pz, 0.5f, 0.5f, 0.0f, h, n, n, n + 1, __fmul_rn(k0, vz));
    scatter_fx(acc + 10 * M, px, py, pz, 0.5f, 0.5f, 0.5f, h, n, n, n, frac);
    scatter_fx(acc + 11 * M, px, py, pz, 0.5f, 0.5f, 0.5f, h, n, n, n, __fmul_rn(frac, S.ptemp[t]));
}

__device__ __forceinline__ bool in_box(const int* b, int i, int j, int k, int grow_hi) {
    return i >= b[0] && j >= b[1] && k >= b[2] && i <= b[3] + grow_hi && j <= b[4] + grow_hi && k <= b[5] + grow_hi;
}

// Obstacle fields of one substep (grid.py:202-213 plus the particle sums): reads and clears the fixed-point
// accumulators, adds the static heater fields, zeroes the wall fluxes (grid.py:62-67).
__device__ __forceinline__ float take(long long* acc, int idx) {
    long long v = acc[idx];
    if (v) acc[idx] = 0;
    return fx_to_float(v);
}

__device__ __forceinline__ float plus_static(float a, const float* st, int idx) {
    return st ? __fadd_rn(a, __ldg(st + idx)) : a;
}

// One cell of the obstacle fields (grid.py:202-213 plus the particle sums; grid.py:62-67 wall fluxes).
__device__ __forceinline__ void obstacle_cell(const hf_scene& S, bool particles, long long* acc, long long M, int t, int i,
                                              int j, int k) {
    const int n = S.n;
    // cell lattices: alpha_s (+ static), alpha and tsum of the heat field
    float a_s = particles ? take(acc, t) : 0.0f;
    S.alpha_s[t] = plus_static(a_s, S.st_alpha, t);
    S.alpha[t] = particles ? take(acc + 10 * M, t) : 0.0f;
    S.tsum[t] = particles ? take(acc + 11 * M, t) : 0.0f;
    // faces: low face of this cell, plus the high wall face on the last layer
    const int fu[2] = {uidx(n, i, j, k), uidx(n, n, j, k)};
    const int fv[2] = {vidx(n, i, j, k), vidx(n, i, n, k)};
    const int fw[2] = {widx(n, i, j, k), widx(n, i, j, n)};
    const bool hi[3] = {i == n - 1, j == n - 1, k == n - 1};
    const bool lo_wall[3] = {i == 0, j == 0, k == 0};
    float* q[3] = {S.qx, S.qy, S.qz};
    float* kf[3] = {S.kx, S.ky, S.kz};
    float* mf[3] = {S.mx, S.my, S.mz};
    const float* stk[3] = {S.st_kx, S.st_ky, S.st_kz};
    const float* stm[3] = {S.st_mx, S.st_my, S.st_mz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int* f = a == 0 ? fu : (a == 1 ? fv : fw);
        for (int side = 0; side < 2; ++side) {
            if (side == 1 && !hi[a]) break;
            const int idx = f[side];
            const bool wall = side == 1 || lo_wall[a];
            float qv = particles ? take(acc + (1 + a) * M, idx) : 0.0f;
            q[a][idx] = wall ? 0.0f : qv;
            float kv = particles ? take(acc + (4 + a) * M, idx) : 0.0f;
            kf[a][idx] = plus_static(kv, stk[a], idx);
            float mv = particles ? take(acc + (7 + a) * M, idx) : 0.0f;
            mf[a][idx] = plus_static(mv, stm[a], idx);
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_obstacle(const hf_scene* __restrict__ scenes, const WorkItem* __restrict__ work,
                                                      int all_scenes) {
    const WorkItem wi = work[blockIdx.x];
    const hf_scene& S = scenes[wi.scene];
    const bool particles = (S.flags & HF_FLAG_PARTICLES) && S.acc != nullptr;
    if (!particles && !all_scenes) return;
    const int n = S.n, N = n * n * n;
    const long long M = (long long)(n + 1) * (n + 1) * (n + 1);
    const int* bnow = S.state->box;
    const int* bprev = S.state->box_prev;
    for (int m = 0; m < kCellsPerThread; ++m) {
        const int t = wi.first + threadIdx.x + m * kThreads;
        if (t >= N) break;
        int i, j, k;
        cell_ijk(t, n, i, j, k);
        // only the particles' footprint of this and the previous substep changes (the rest holds the static fields)
        if (!all_scenes && !in_box(bnow, i, j, k, 0) && !in_box(bprev, i, j, k, 0)) continue;
        obstacle_cell(S, particles, S.acc, M, t, i, j, k);
    }
}

// The bounding box of this and the previous substep's footprints grown by `grow` and clamped to the grid; false when
// both are empty.  Every cell of it may be recomputed: outside the footprints the accumulators are zero and the
// fields equal the statics, so a recomputation reproduces them.
__device__ __forceinline__ bool footprint_union(const hf_scene& S, int grow, int (&lo)[3], int (&hi)[3]) {
    const int* a = S.state->box;
    const int* b = S.state->box_prev;
    const bool ea = a[0] > a[3], eb = b[0] > b[3];
    if (ea && eb) return false;
    for (int d = 0; d < 3; ++d) {
        lo[d] = max(0, (ea ? b[d] : eb ? a[d] : min(a[d], b[d])) - grow);
        hi[d] = min(S.n - 1, (ea ? b[3 + d] : eb ? a[3 + d] : max(a[3 + d], b[3 + d])) + grow);
    }
    return true;
}

// k_obstacle for one coupled scene over the footprint union only (the substep's rebuild)
__global__ void __launch_bounds__(kThreads) k_obstacle_box(const hf_scene* __restrict__ scenes, int s) {
    const hf_scene& S = scenes[s];
    int lo[3], hi[3];
    if (!footprint_union(S, 0, lo, hi)) return;
    const int n = S.n;
    const long long M = (long long)(n + 1) * (n + 1) * (n + 1);
    const int ei = hi[0] - lo[0] + 1, ej = hi[1] - lo[1] + 1, ek = hi[2] - lo[2] + 1;
    const int cells = ei * ej * ek;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < cells; q += gridDim.x * blockDim.x) {
        const int k = lo[2] + q % ek, j = lo[1] + (q / ek) % ej, i = lo[0] + q / (ek * ej);
        obstacle_cell(S, true, S.acc, M, (i * n + j) * n + k, i, j, k);
    }
}

// grid.py:46-59 (k_face_fraction) and heat.py:44-47 (k_conductivity) from the obstacle fields, plus the harmonic face
// diffusivity of every interior face (heat.py:50-52; the same value from either side, bit for bit).  The conductivity
// of the lower neighbour is recomputed from its alpha_s (a pure function of it) instead of read, so no cell waits on
// another thread.  Coupled scenes rebuild only their particle footprint grown by one cell on the high side.
__device__ __forceinline__ float conductivity(float a, float ka, float km) {
    return __fadd_rn(ka, __fmul_rn(__fsub_rn(km, ka), clampf_(__fdiv_rn(a, 0.6f), 0.0f, 1.0f)));
}

// One cell of the coefficient stage: conductivity (heat.py:44-47), face fractions (grid.py:46-59) and face
// diffusivities (heat.py:50-53) of the cell's low faces (and the high wall faces on the last layer).
__device__ __forceinline__ void coeff_cell(const hf_scene& S, float afmin, float ka, float km, const float* as, int t,
                                           int i, int j, int k) {
    const int n = S.n;
    const float ac = as[t];
    const float kc = conductivity(ac, ka, km);
    S.kap[t] = kc;
    const int fu = uidx(n, i, j, k), fv = vidx(n, i, j, k), fw = widx(n, i, j, k);
    if (i == 0) {
        S.ax[fu] = 0.0f;
        S.hkx[fu] = 0.0f;
    } else {
        const float an = as[t - n * n];
        S.ax[fu] = clampf_(__fsub_rn(1.0f, __fmul_rn(0.5f, __fadd_rn(an, ac))), afmin, 1.0f);
        S.hkx[fu] = face_kappa(conductivity(an, ka, km), kc);
    }
    float ayv = 0.0f, azv = 0.0f;
    if (j == 0) {
        S.hky[fv] = 0.0f;
    } else {
        const float an = as[t - n];
        ayv = clampf_(__fsub_rn(1.0f, __fmul_rn(0.5f, __fadd_rn(an, ac))), afmin, 1.0f);
        S.hky[fv] = face_kappa(conductivity(an, ka, km), kc);
    }
    float hkzv = 0.0f;
    if (k != 0) {
        const float an = as[t - 1];
        azv = clampf_(__fsub_rn(1.0f, __fmul_rn(0.5f, __fadd_rn(an, ac))), afmin, 1.0f);
        hkzv = face_kappa(conductivity(an, ka, km), kc);
    }
    S.hkz[fw] = hkzv;
    if (S.hkzc) S.hkzc[t] = hkzv;   // cell-layout copy for the tiled (TMA) heat stencil
    S.ay[fv] = ayv;
    S.az[fw] = azv;
    S.ayc[t] = ayv;   // cell-layout copies for the tiled (TMA) pressure stencil
    S.azc[t] = azv;
    if (i == n - 1) S.ax[uidx(n, n, j, k)] = S.hkx[uidx(n, n, j, k)] = 0.0f;
    if (j == n - 1) S.ay[vidx(n, i, n, k)] = S.hky[vidx(n, i, n, k)] = 0.0f;
    if (k == n - 1) S.az[widx(n, i, j, n)] = S.hkz[widx(n, i, j, n)] = 0.0f;
}

__global__ void __launch_bounds__(kThreads) k_coeff(const hf_scene* __restrict__ scenes, const WorkItem* __restrict__ work,
                                                   int all_scenes) {
    const WorkItem wi = work[blockIdx.x];
    const hf_scene& S = scenes[wi.scene];
    if (!all_scenes && !(S.flags & HF_FLAG_PARTICLES)) return;
    const int n = S.n, N = n * n * n;
    const float afmin = (float)S.alpha_f_min, ka = (float)S.kappa_air, km = (float)S.kappa_mat;
    const int* bnow = S.state->box;
    const int* bprev = S.state->box_prev;
    for (int m = 0; m < kCellsPerThread; ++m) {
        const int t = wi.first + threadIdx.x + m * kThreads;
        if (t >= N) break;
        int i, j, k;
        cell_ijk(t, n, i, j, k);
        if (!all_scenes && !in_box(bnow, i, j, k, 1) && !in_box(bprev, i, j, k, 1)) continue;
        coeff_cell(S, afmin, ka, km, S.alpha_s, t, i, j, k);
    }
}

// k_coeff for one coupled scene over the footprint union grown by one cell (the substep's rebuild)
__global__ void __launch_bounds__(kThreads) k_coeff_box(const hf_scene* __restrict__ scenes, int s) {
    const hf_scene& S = scenes[s];
    int lo[3], hi[3];
    if (!footprint_union(S, 1, lo, hi)) return;
    const int n = S.n;
    const float afmin = (float)S.alpha_f_min, ka = (float)S.kappa_air, km = (float)S.kappa_mat;
    const int ei = hi[0] - lo[0] + 1, ej = hi[1] - lo[1] + 1, ek = hi[2] - lo[2] + 1;
    const int cells = ei * ej * ek;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < cells; q += gridDim.x * blockDim.x) {
        const int k = lo[2] + q % ek, j = lo[1] + (q / ek) % ej, i = lo[0] + q / (ek * ej);
        coeff_cell(S, afmin, ka, km, S.alpha_s, (i * n + j) * n + k, i, j, k);
    }
}

// --------------------------------------------------------------------------------------------- temperature
// solver.py:74-77: k_blend (heat.py:21-28), k_apply_fixed (heat.py:147-151), k_source (heat.py:154-158) -> Tw
__global__ void __launch_bounds__(kThreads) k_prestage(const hf_scene* __restrict__ scenes, const WorkItem* __restrict__ work,
                                                      double dt_d) {
    const WorkItem wi = work[blockIdx.x];
    const hf_scene& S = scenes[wi.scene];
    const int n = S.n, N = n * n * n;
    const int par = S.state->parity;
    const float* T = S.T[par];
    const bool source = (S.flags & HF_FLAG_SOURCE) != 0, particles = (S.flags & HF_FLAG_PARTICLES) != 0;
    const float rate = (float)S.rate, t_cap = (float)S.t_cap, dt = (float)dt_d;
    for (int m = 0; m < kCellsPerThread; ++m) {
        const int t = wi.first + threadIdx.x + m * kThreads;
        if (t >= N) break;
        float tw;
        if (particles) {
            const float a = S.alpha[t];
            tw = a > 0.05f ? __fdiv_rn(S.tsum[t], a) : T[t];
        } else {
            tw = T[t];   // alpha = 0 everywhere without particles: k_blend keeps T
        }
        const uint8_t fl = S.cell_flags[t];
        if (fl & 1) tw = S.tfix[t];
        if (source && (fl & 2)) tw = minf_(__fadd_rn(tw, __fmul_rn(rate, dt)), maxf_(tw, t_cap));
        S.Tw[t] = tw;
    }
}

// heat.py:161-174 k_particle_update: FLIP increment between Tw and the diffused T, melt law
__global__ void __launch_bounds__(kThreads) k_particle_update(const hf_scene* __restrict__ scenes, int s) {
    const hf_scene& S = scenes[s];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) {
        // the footprint of this substep becomes the previous one; the next scatter starts from an empty box
        hf_scene_state* st = S.state;
#pragma unroll
        for (int d = 0; d < 6; ++d) st->box_prev[d] = st->box[d];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            st->box[d] = INT_MAX;
            st->box[3 + d] = INT_MIN;
        }
    }
    if (t >= S.n_particles) return;
    const int n = S.n, par = S.state->parity;
    const float h = (float)S.h;
    const float t_sol = (float)S.t_sol, t_liq = (float)S.t_liq, y_solid = (float)S.y_solid;
    const float mu_s = (float)S.mu_s, mu_l = (float)S.mu_l, t_max = (float)S.t_max;
    const float px = S.pos[3 * t], py = S.pos[3 * t + 1], pz = S.pos[3 * t + 2];
    const GridPos q = grid_pos(px, py, pz, div_by(h));
    const float dT = __fsub_rn(sample_at(S.T[par ^ 1], q, 0.5f, 0.5f, 0.5f, n, n, n),
                               sample_at(S.Tw, q, 0.5f, 0.5f, 0.5f, n, n, n));
    const float tp = clampf_(__fadd_rn(S.ptemp[t], dT), 0.0f, t_max);
    S.ptemp[t] = tp;
    const float f = clampf_(__fdiv_rn(__fsub_rn(tp, t_sol), __fsub_rn(t_liq, t_sol)), 0.0f, 1.0f);
    S.pmelt[t] = f;
    S.pyield[t] = __fmul_rn(y_solid, __fsub_rn(1.0f, f));
    S.pvisc[t] = __fadd_rn(__fmul_rn(mu_s, __fsub_rn(1.0f, f)), __fmul_rn(mu_l, f));
}

// ------------------------------------------------------------------------------------------------ air faces
// grid.py:219-233 for the faces of one cell: k_advect_face from the old u,v,w (grid.py:25-33), k_buoyancy on w
// (grid.py:36-43, with the new T), k_relax (grid.py:70-79).  Each face's value depends only on its own intermediate
// values, so applying the three kernels face by face is the same arithmetic as the reference's three passes.
__device__ __forceinline__ float relax_face(float q, float af, float kf, float mf, float rho, float afmin, float h,
                                            float dt) {
    // 1 / (...) correctly rounded: __frcp_rn is the IEEE round-to-nearest reciprocal, the same value as __fdiv_rn(1, .)
    const float c = __frcp_rn(__fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(rho, maxf_(af, afmin)), h), h), h));
    const float dtc = __fmul_rn(dt, c);
    return __fdiv_rn(__fadd_rn(q, __fmul_rn(dtc, mf)), __fadd_rn(1.0f, __fmul_rn(dtc, kf)));
}

// ------------------------------------------------------------------- face stage from staged velocity boxes
// The face stage per CG tile (4 x 8 x 32 cells, 512 threads, two cells per thread): the old u, v, w around the tile are
// staged in shared memory as boxes with a kFH-cell halo whose entries outside the lattice repeat the nearest lattice
// node.  A trilinear sample whose eight nodes fall in the box then reads box[lower - origin] and its +1 neighbours,
// which hold lattice[clamp(lower)] and lattice[clamp(lower + 1)] -- exactly the nodes fields.py:16-28 reads after
// clamping -- with 32-bit shared addresses and no clamps; a sample outside the box (a back-trace longer than the halo)
// reads the lattice itself.  Positions, weights and the order of every operation are those of sample_at, so the
// results are the same bits as sampling the lattice directly (fields.py's clamped nodes).
constexpr int kFH = 2;
constexpr int kFBX = kTI + 2 * kFH + 1, kFBY = kTJ + 2 * kFH + 1, kFBZ = kTK + 2 * kFH + 1;   // 9 x 13 x 37
constexpr int kFBox = kFBX * kFBY * kFBZ;
constexpr int kFaceThreads = 512;
constexpr size_t kFaceSmem = 3 * (size_t)kFBox * sizeof(float);

// one axis of a sample: unclamped lower node i (box-local: i - origin), weights w0 = 1 - f and f (fields.py:14-27)
struct BAxis {
    int i, b;
    float w0, f;
};

__device__ __forceinline__ BAxis baxis(float q, float off, int origin) {
    const float g = __fsub_rn(q, off);
    const int i = (int)floorf(g);
    const float f = __fsub_rn(g, (float)i);
    return BAxis{i, i - origin, __fsub_rn(1.0f, f), f};
}

__device__ __forceinline__ bool in_box(const BAxis& X, const BAxis& Y, const BAxis& Z) {
    return (unsigned)X.b <= (unsigned)(kFBX - 2) && (unsigned)Y.b <= (unsigned)(kFBY - 2) &&
           (unsigned)Z.b <= (unsigned)(kFBZ - 2);
}

// sample_at's eight terms in its order (fields.py:29-35: weight ((wx * wy) * wz) * a, dx, dy, dz), from a box or
// (outside it) from the lattice with the clamped nodes
__device__ __forceinline__ float box_sample(const float* __restrict__ B, const float* __restrict__ a, const BAxis& X,
                                            const BAxis& Y, const BAxis& Z, int nx, int ny, int nz) {
    float v[8];
    if (in_box(X, Y, Z)) {
        const float* c = B + (X.b * kFBY + Y.b) * kFBZ + Z.b;
        v[0] = c[0];
        v[1] = c[1];
        v[2] = c[kFBZ];
        v[3] = c[kFBZ + 1];
        v[4] = c[kFBY * kFBZ];
        v[5] = c[kFBY * kFBZ + 1];
        v[6] = c[kFBY * kFBZ + kFBZ];
        v[7] = c[kFBY * kFBZ + kFBZ + 1];
    } else {
        const int x0 = clampi(X.i, 0, nx - 1), x1 = clampi(X.i + 1, 0, nx - 1);
        const int y0 = clampi(Y.i, 0, ny - 1), y1 = clampi(Y.i + 1, 0, ny - 1);
        const int z0 = clampi(Z.i, 0, nz - 1), z1 = clampi(Z.i + 1, 0, nz - 1);
        const int sy = nz, sx = ny * nz;
        v[0] = __ldg(a + x0 * sx + y0 * sy + z0);
        v[1] = __ldg(a + x0 * sx + y0 * sy + z1);
        v[2] = __ldg(a + x0 * sx + y1 * sy + z0);
        v[3] = __ldg(a + x0 * sx + y1 * sy + z1);
        v[4] = __ldg(a + x1 * sx + y0 * sy + z0);
        v[5] = __ldg(a + x1 * sx + y0 * sy + z1);
        v[6] = __ldg(a + x1 * sx + y1 * sy + z0);
        v[7] = __ldg(a + x1 * sx + y1 * sy + z1);
    }
    float s = 0.0f;
    s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fmul_rn(X.w0, Y.w0), Z.w0), v[0]));
    s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fmul_rn(X.w0, Y.w0), Z.f), v[1]));
    s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fmul_rn(X.w0, Y.f), Z.w0), v[2]));
    s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fmul_rn(X.w0, Y.f), Z.f), v[3]));
    s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fmul_rn(X.f, Y.w0), Z.w0), v[4]));
    s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fmul_rn(X.f, Y.w0), Z.f), v[5]));
    s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fmul_rn(X.f, Y.f), Z.w0), v[6]));
    s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fmul_rn(X.f, Y.f), Z.f), v[7]));
    return s;
}

// sample_velocity (fields.py:68-72) from the boxes: the three lattices at one point
__device__ __forceinline__ void box_velocity(const float* Bu, const float* Bv, const float* Bw, const float* __restrict__ u,
                                             const float* __restrict__ v, const float* __restrict__ w, float px,
                                             float py, float pz, const DivBy& h, int n, int ox, int oy, int oz, float* o) {
    const GridPos q = grid_pos(px, py, pz, h);
    const BAxis x0 = baxis(q.x, 0.0f, ox), x5 = baxis(q.x, 0.5f, ox);
    const BAxis y0 = baxis(q.y, 0.0f, oy), y5 = baxis(q.y, 0.5f, oy);
    const BAxis z0 = baxis(q.z, 0.0f, oz), z5 = baxis(q.z, 0.5f, oz);
    o[0] = box_sample(Bu, u, x0, y5, z5, n + 1, n, n);
    o[1] = box_sample(Bv, v, x5, y0, z5, n, n + 1, n);
    o[2] = box_sample(Bw, w, x5, y5, z0, n, n, n + 1);
}

// backtrace (fields.py:111-116) from the boxes
__device__ __forceinline__ void box_backtrace(const float* Bu, const float* Bv, const float* Bw, const float* __restrict__ u,
                                              const float* __restrict__ v, const float* __restrict__ w, const float* x,
                                              const DivBy& h, int n, float dt, int ox, int oy, int oz, float* o) {
    float vel[3];
    box_velocity(Bu, Bv, Bw, u, v, w, x[0], x[1], x[2], h, n, ox, oy, oz, vel);
    const float hdt = __fmul_rn(0.5f, dt);
    const float y0 = __fsub_rn(x[0], __fmul_rn(hdt, vel[0]));
    const float y1 = __fsub_rn(x[1], __fmul_rn(hdt, vel[1]));
    const float y2 = __fsub_rn(x[2], __fmul_rn(hdt, vel[2]));
    box_velocity(Bu, Bv, Bw, u, v, w, y0, y1, y2, h, n, ox, oy, oz, vel);
    o[0] = __fsub_rn(x[0], __fmul_rn(dt, vel[0]));
    o[1] = __fsub_rn(x[1], __fmul_rn(dt, vel[1]));
    o[2] = __fsub_rn(x[2], __fmul_rn(dt, vel[2]));
}

// sample (fields.py:5-36) of one lattice with offsets (offx, offy, offz) from its box
__device__ __forceinline__ float box_point(const float* B, const float* __restrict__ a, const float* y, float offx,
                                           float offy, float offz, const DivBy& h, int nx, int ny, int nz, int ox, int oy,
                                           int oz) {
    const GridPos q = grid_pos(y[0], y[1], y[2], h);
    return box_sample(B, a, baxis(q.x, offx, ox), baxis(q.y, offy, oy), baxis(q.z, offz, oz), nx, ny, nz);
}

// grid.py:219-233 for the faces of the cells of one CG tile (relax_face's fused per-face arithmetic, sampling from the
// staged boxes); block = 512 threads, thread lt owns cells (i0 + 2 (lt / 256) + {0, 1}, j0 + (lt % 256) / 32, k0 + lt % 32).
__global__ void __launch_bounds__(kFaceThreads, 2) k_face_tile(const hf_scene* __restrict__ scenes,
                                                              const TileItem* __restrict__ tiles, double dt_d) {
    extern __shared__ float fbox[];
    const TileItem ti = tiles[blockIdx.x];
    const hf_scene& S = scenes[ti.scene];
    const int n = S.n;
    const int par = S.state->parity;
    const float *u0 = S.u[par], *v0 = S.v[par], *w0 = S.w[par];
    float *u1 = S.u[par ^ 1], *v1 = S.v[par ^ 1], *w1 = S.w[par ^ 1];
    const float* Tn = S.T[par ^ 1];
    const float h = (float)S.h, dt = (float)dt_d, rho = (float)S.rho, afmin = (float)S.alpha_f_min;
    const float g = (float)S.g, t_amb = (float)S.t_amb;
    const bool buoy = (S.flags & HF_FLAG_BUOYANCY) != 0;
    const float buoy_num = __fmul_rn(dt, g);
    const DivBy hd = div_by(h), buoy_den = div_by(__fadd_rn(t_amb, 273.15f));
    float* Bu = fbox;
    float* Bv = fbox + kFBox;
    float* Bw = fbox + 2 * kFBox;
    const int ox = ti.i0 - kFH, oy = ti.j0 - kFH, oz = ti.k0 - kFH;
    // the boxes: lattice node (ox + a, oy + b, oz + c), clamped to the lattice
    for (int e = threadIdx.x; e < kFBox; e += kFaceThreads) {
        const int a = e / (kFBY * kFBZ), r = e - a * (kFBY * kFBZ), b = r / kFBZ, c = r - b * kFBZ;
        const int gi = ox + a, gj = oy + b, gk = oz + c;
        const int iu = clampi(gi, 0, n), ic = clampi(gi, 0, n - 1);
        const int ju = clampi(gj, 0, n), jc = clampi(gj, 0, n - 1);
        const int ku = clampi(gk, 0, n), kc = clampi(gk, 0, n - 1);
        Bu[e] = __ldg(u0 + (iu * n + jc) * n + kc);               // (n+1, n, n)
        Bv[e] = __ldg(v0 + (ic * (n + 1) + ju) * n + kc);         // (n, n+1, n)
        Bw[e] = __ldg(w0 + (ic * n + jc) * (n + 1) + ku);         // (n, n, n+1)
    }
    __syncthreads();
    const int lt = threadIdx.x & 255;
    const int j = ti.j0 + (lt >> 5), k = ti.k0 + (lt & 31);
    if (j >= n || k >= n) return;
    for (int mm = 0; mm < 2; ++mm) {
        const int i = ti.i0 + 2 * (threadIdx.x >> 8) + mm;
        if (i >= n) break;
        const int t = (i * n + j) * n + k;
        const float fi = (float)i, fj = (float)j, fk = (float)k;
        const float ci = __fmul_rn(__fadd_rn(fi, 0.5f), h), cj = __fmul_rn(__fadd_rn(fj, 0.5f), h),
                    ck = __fmul_rn(__fadd_rn(fk, 0.5f), h);
        float y[3];
        // u(i,j,k)
        {
            const int f = uidx(n, i, j, k);
            float val = 0.0f;
            if (i != 0) {
                const float x[3] = {__fmul_rn(fi, h), cj, ck};
                box_backtrace(Bu, Bv, Bw, u0, v0, w0, x, hd, n, dt, ox, oy, oz, y);
                val = box_point(Bu, u0, y, 0.0f, 0.5f, 0.5f, hd, n + 1, n, n, ox, oy, oz);
                val = relax_face(val, S.ax[f], S.kx[f], S.mx[f], rho, afmin, h, dt);
            }
            u1[f] = val;
            if (i == n - 1) u1[uidx(n, n, j, k)] = 0.0f;
        }
        // v(i,j,k)
        {
            const int f = vidx(n, i, j, k);
            float val = 0.0f;
            if (j != 0) {
                const float x[3] = {ci, __fmul_rn(fj, h), ck};
                box_backtrace(Bu, Bv, Bw, u0, v0, w0, x, hd, n, dt, ox, oy, oz, y);
                val = box_point(Bv, v0, y, 0.5f, 0.0f, 0.5f, hd, n, n + 1, n, ox, oy, oz);
                val = relax_face(val, S.ay[f], S.ky[f], S.my[f], rho, afmin, h, dt);
            }
            v1[f] = val;
            if (j == n - 1) v1[vidx(n, i, n, k)] = 0.0f;
        }
        // w(i,j,k)
        {
            const int f = widx(n, i, j, k);
            float val = 0.0f;
            if (k != 0) {
                const float x[3] = {ci, cj, __fmul_rn(fk, h)};
                box_backtrace(Bu, Bv, Bw, u0, v0, w0, x, hd, n, dt, ox, oy, oz, y);
                val = box_point(Bw, w0, y, 0.5f, 0.5f, 0.0f, hd, n, n, n + 1, ox, oy, oz);
                if (buoy) {
                    const float tf = __fmul_rn(0.5f, __fadd_rn(Tn[t - 1], Tn[t]));
                    val = __fadd_rn(val, div_rn(__fmul_rn(buoy_num, __fsub_rn(tf, t_amb)), buoy_den));
                }
                val = relax_face(val, S.az[f], S.kz[f], S.mz[f], rho, afmin, h, dt);
            }
            w1[f] = val;
            if (k == n - 1) w1[widx(n, i, j, n)] = 0.0f;
        }
    }
}

size_t face_tile_smem() { return kFaceSmem; }

// solver.py:78 k_advect (heat.py:31-41) into T[parity^1], fused with k_heat_rhs (heat.py:108-118), per CG tile: the
// old u, v, w and Tw around the tile staged in shared memory as in k_face_tile (the same bits as sampling the
// lattices directly).  512 threads, two cells per thread.
__global__ void __launch_bounds__(kFaceThreads, 2) k_advect_T_tile(const hf_scene* __restrict__ scenes,
                                                                  const TileItem* __restrict__ tiles, double dt_d) {
    extern __shared__ float fbox[];
    const TileItem ti = tiles[blockIdx.x];
    const hf_scene& S = scenes[ti.scene];
    const int n = S.n;
    const int par = S.state->parity;
    const float *u = S.u[par], *v = S.v[par], *w = S.w[par];
    float* T2 = S.T[par ^ 1];
    const float h = (float)S.h, dt = (float)dt_d;
    const float* Tw = S.Tw;
    const uint8_t* fl = S.cell_flags;
    const float c_dt = __fdiv_rn(dt, __fmul_rn(h, h));
    const DivBy hd = div_by(h);
    float* Bu = fbox;
    float* Bv = fbox + kFBox;
    float* Bw = fbox + 2 * kFBox;
    float* BT = fbox + 3 * kFBox;
    const int ox = ti.i0 - kFH, oy = ti.j0 - kFH, oz = ti.k0 - kFH;
    for (int e = threadIdx.x; e < kFBox; e += kFaceThreads) {
        const int a = e / (kFBY * kFBZ), r = e - a * (kFBY * kFBZ), b = r / kFBZ, c = r - b * kFBZ;
        const int gi = ox + a, gj = oy + b, gk = oz + c;
        const int iu = clampi(gi, 0, n), ic = clampi(gi, 0, n - 1);
        const int ju = clampi(gj, 0, n), jc = clampi(gj, 0, n - 1);
        const int ku = clampi(gk, 0, n), kc = clampi(gk, 0, n - 1);
        Bu[e] = __ldg(u + (iu * n + jc) * n + kc);                // (n+1, n, n)
        Bv[e] = __ldg(v + (ic * (n + 1) + ju) * n + kc);          // (n, n+1, n)
        Bw[e] = __ldg(w + (ic * n + jc) * (n + 1) + ku);          // (n, n, n+1)
        BT[e] = __ldg(Tw + (ic * n + jc) * n + kc);               // (n, n, n)
    }
    __syncthreads();
    const int lt = threadIdx.x & 255;
    const int j = ti.j0 + (lt >> 5), k = ti.k0 + (lt & 31);
    if (j >= n || k >= n) return;
    for (int mm = 0; mm < 2; ++mm) {
        const int i = ti.i0 + 2 * (threadIdx.x >> 8) + mm;
        if (i >= n) break;
        const int t = (i * n + j) * n + k;
        // the heat rhs's flags and face diffusivities are loaded first (in bounds: a missing neighbour reads the cell
        // itself, the face lattices have n + 1 layers), so they arrive while the back-trace is computed
        const int nbr[6] = {t - n * n, t + n * n, t - n, t + n, t - 1, t + 1};
        const bool in[6] = {i > 0, i < n - 1, j > 0, j < n - 1, k > 0, k < n - 1};
        const uint8_t fc = fl[t];
        uint8_t fn[6];
        float kf[6];
        const float* hk[6] = {S.hkx + uidx(n, i, j, k), S.hkx + uidx(n, i + 1, j, k), S.hky + vidx(n, i, j, k),
                              S.hky + vidx(n, i, j + 1, k), S.hkz + widx(n, i, j, k), S.hkz + widx(n, i, j, k + 1)};
#pragma unroll
        for (int s = 0; s < 6; ++s) {
            fn[s] = fl[in[s] ? nbr[s] : t];
            kf[s] = *hk[s];
        }
        float out;
        if (S.alpha_s[t] > 0.5f) {
            out = Tw[t];
        } else {
            const float x[3] = {__fmul_rn(__fadd_rn((float)i, 0.5f), h), __fmul_rn(__fadd_rn((float)j, 0.5f), h),
                                __fmul_rn(__fadd_rn((float)k, 0.5f), h)};
            float y[3];
            box_backtrace(Bu, Bv, Bw, u, v, w, x, hd, n, dt, ox, oy, oz, y);
            out = box_point(BT, Tw, y, 0.5f, 0.5f, 0.5f, hd, n, n, n, ox, oy, oz);
        }
        T2[t] = out;
        // heat rhs: tfix on fixed cells, else T2 + dt/h^2 * sum over fixed neighbours of kappa_f * tfix
        float rhs;
        if (fc & 1) {
            rhs = S.tfix[t];
        } else {
            float acc = 0.0f;
#pragma unroll
            for (int s = 0; s < 6; ++s) {
                if (!in[s]) continue;
                if (fn[s] & 1) acc = __fadd_rn(acc, __fmul_rn(kf[s], S.tfix[nbr[s]]));
            }
            rhs = __fadd_rn(out, __fmul_rn(c_dt, acc));
        }
        S.hrhs[t] = rhs;
    }
}

size_t advect_tile_smem() { return 4 * (size_t)kFBox * sizeof(float); }

// grid.py:82-91 k_divergence_rhs with scale rho/dt into rhs, plus the fp64 partial sum of the chunk for the mean of
// grid.py:238-241 (reduced over the scene by the pressure CG kernel, in a fixed tree).
__global__ void __launch_bounds__(kChunk) k_divergence(const hf_scene* __restrict__ scenes, const WorkItem* __restrict__ work,
                                                     double dt_d, Workspace ws) {
    // one cell per thread (1024 per chunk, so all of a cell's loads are in flight at once); the chunk's sum is then
    // formed in the tree of a 256-thread pass -- thread lt adds cells lt, lt + 256, lt + 512, lt + 768 in order, warp
    // butterfly, 8 warps in order -- from the values parked in shared memory
    __shared__ float rv[kChunk];
    __shared__ double red[kThreads / 32];
    const int c = blockIdx.x;
    const WorkItem wi = work[c];
    const hf_scene& S = scenes[wi.scene];
    const int n = S.n, N = n * n * n;
    const int par = S.state->parity;
    const float *u = S.u[par ^ 1], *v = S.v[par ^ 1], *w = S.w[par ^ 1];
    const float h = (float)S.h, scale = (float)(S.rho / dt_d);
    const int t = wi.first + threadIdx.x;
    if (t < N) {
        int i, j, k;
        cell_ijk(t, n, i, j, k);
        const int u0 = uidx(n, i, j, k), u1i = uidx(n, i + 1, j, k);
        const int v0 = vidx(n, i, j, k), v1i = vidx(n, i, j + 1, k);
        const int w0 = widx(n, i, j, k), w1i = w0 + 1;
        float d = __fmul_rn(S.ax[u1i], u[u1i]);
        d = __fadd_rn(d, S.qx[u1i]);
        d = __fsub_rn(d, __fmul_rn(S.ax[u0], u[u0]));
        d = __fsub_rn(d, S.qx[u0]);
        d = __fadd_rn(d, __fmul_rn(S.ay[v1i], v[v1i]));
        d = __fadd_rn(d, S.qy[v1i]);
        d = __fsub_rn(d, __fmul_rn(S.ay[v0], v[v0]));
        d = __fsub_rn(d, S.qy[v0]);
        d = __fadd_rn(d, __fmul_rn(S.az[w1i], w[w1i]));
        d = __fadd_rn(d, S.qz[w1i]);
        d = __fsub_rn(d, __fmul_rn(S.az[w0], w[w0]));
        d = __fsub_rn(d, S.qz[w0]);
        d = __fdiv_rn(d, h);
        const float r = __fmul_rn(-scale, d);
        S.rhs[t] = r;
        rv[threadIdx.x] = r;
    }
    __syncthreads();
    if (threadIdx.x < kThreads) {
        double part = 0.0;
#pragma unroll
        for (int m = 0; m < kCellsPerThread; ++m) {
            if (wi.first + threadIdx.x + m * kThreads >= N) break;
            part += (double)rv[threadIdx.x + m * kThreads];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < kThreads / 32; ++q) s += red[q];
        ws.mean_part[c] = s;
    }
}

// ---------------------------------------------------------------------------------------------- diagnostics
// grid.py:156-162 k_cell_velocity
__global__ void k_cell_velocity(const hf_scene* __restrict__ scenes, int s, float* __restrict__ out) {
    const hf_scene& S = scenes[s];
    const int n = S.n, N = n * n * n, par = S.state->parity;
    const float *u = S.u[par], *v = S.v[par], *w = S.w[par];
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < N; t += gridDim.x * blockDim.x) {
        int i, j, k;
        cell_ijk(t, n, i, j, k);
        out[3 * t + 0] = __fmul_rn(0.5f, __fadd_rn(u[uidx(n, i, j, k)], u[uidx(n, i + 1, j, k)]));
        out[3 * t + 1] = __fmul_rn(0.5f, __fadd_rn(v[vidx(n, i, j, k)], v[vidx(n, i, j + 1, k)]));
        out[3 * t + 2] = __fmul_rn(0.5f, __fadd_rn(w[widx(n, i, j, k)], w[widx(n, i, j, k) + 1]));
    }
}

// grid.py:257-260 divergence_max (k_divergence_rhs with scale 1, max |.| * h) and grid.py:262-263 speed_max.
// Non-negative floats order like their bit patterns, so atomicMax on the bits gives the maximum.
__global__ void k_divergence_max(const hf_scene* __restrict__ scenes, int s, unsigned* __restrict__ out_bits) {
    const hf_scene& S = scenes[s];
    const int n = S.n, N = n * n * n, par = S.state->parity;
    const float *u = S.u[par], *v = S.v[par], *w = S.w[par];
    const float h = (float)S.h;
    float mx = 0.0f;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < N; t += gridDim.x * blockDim.x) {
        int i, j, k;
        cell_ijk(t, n, i, j, k);
        const int u0 = uidx(n, i, j, k), u1i = uidx(n, i + 1, j, k);
        const int v0 = vidx(n, i, j, k), v1i = vidx(n, i, j + 1, k);
        const int w0 = widx(n, i, j, k), w1i = w0 + 1;
        float d = __fmul_rn(S.ax[u1i], u[u1i]);
        d = __fadd_rn(d, S.qx[u1i]);
        d = __fsub_rn(d, __fmul_rn(S.ax[u0], u[u0]));
        d = __fsub_rn(d, S.qx[u0]);
        d = __fadd_rn(d, __fmul_rn(S.ay[v1i], v[v1i]));
        d = __fadd_rn(d, S.qy[v1i]);
        d = __fsub_rn(d, __fmul_rn(S.ay[v0], v[v0]));
        d = __fsub_rn(d, S.qy[v0]);
        d = __fadd_rn(d, __fmul_rn(S.az[w1i], w[w1i]));
        d = __fadd_rn(d, S.qz[w1i]);
        d = __fsub_rn(d, __fmul_rn(S.az[w0], w[w0]));
        d = __fsub_rn(d, S.qz[w0]);
        d = __fdiv_rn(d, h);
        mx = fmaxf(mx, fabsf(__fmul_rn(-1.0f, d)));
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out_bits, __float_as_uint(mx));
}

__global__ void k_speed_max(const hf_scene* __restrict__ scenes, int s, unsigned* __restrict__ out_bits) {
    const hf_scene& S = scenes[s];
    const int n = S.n, par = S.state->parity;
    const int NF = (n + 1) * n * n;
    float mx = 0.0f;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < NF; t += gridDim.x * blockDim.x)
        mx = fmaxf(mx, fmaxf(fabsf(S.u[par][t]), fmaxf(fabsf(S.v[par][t]), fabsf(S.w[par][t]))));
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out_bits, __float_as_uint(mx));
}

// ------------------------------------------------------------------------------------- single-kernel parity
// the constant-divisor division of the sampling stages, elementwise (checked against IEEE division)
__global__ void k_divide_by(int count, const float* __restrict__ x, float y, float* __restrict__ out) {
    const DivBy d = div_by(y);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) out[i] = div_rn(x[i], d);
}

// grid.py:94-115 k_laplacian on plain arrays
__global__ void k_laplacian_plain(int n, float h, float alpha, float beta, const float* __restrict__ p,
                                  const float* __restrict__ ax, const float* __restrict__ ay, const float* __restrict__ az,
                                  const float* __restrict__ y, float* __restrict__ out) {
    const int N = n * n * n, nn = n * n;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < N; t += gridDim.x * blockDim.x) {
        int i, j, k;
        cell_ijk(t, n, i, j, k);
        const float pc = p[t];
        float acc = 0.0f;
        if (i > 0) acc = __fadd_rn(acc, __fmul_rn(ax[uidx(n, i, j, k)], __fsub_rn(pc, p[t - nn])));
        if (i < n - 1) acc = __fadd_rn(acc, __fmul_rn(ax[uidx(n, i + 1, j, k)], __fsub_rn(pc, p[t + nn])));
        if (j > 0) acc = __fadd_rn(acc, __fmul_rn(ay[vidx(n, i, j, k)], __fsub_rn(pc, p[t - n])));
        if (j < n - 1) acc = __fadd_rn(acc, __fmul_rn(ay[vidx(n, i, j + 1, k)], __fsub_rn(pc, p[t + n])));
        if (k > 0) acc = __fadd_rn(acc, __fmul_rn(az[widx(n, i, j, k)], __fsub_rn(pc, p[t - 1])));
        if (k < n - 1) acc = __fadd_rn(acc, __fmul_rn(az[widx(n, i, j, k + 1)], __fsub_rn(pc, p[t + 1])));
        out[t] = __fadd_rn(__fdiv_rn(__fmul_rn(alpha, acc), __fmul_rn(h, h)), __fmul_rn(beta, y[t]));
    }
}

// heat.py:94-105 k_heat_matvec on plain arrays
__global__ void k_heat_matvec_plain(int n, float h, float dt, float alpha, float beta, const float* __restrict__ x,
                                    const float* __restrict__ kap, const uint8_t* __restrict__ fl,
                                    const float* __restrict__ y, float* __restrict__ out) {
    const int N = n * n * n, nn = n * n;
    const float c_dt = __fdiv_rn(dt, __fmul_rn(h, h));
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < N; t += gridDim.x * blockDim.x) {
        int i, j, k;
        cell_ijk(t, n, i, j, k);
        const float xc = x[t];
        if (fl[t] & 1) {
            out[t] = __fadd_rn(__fmul_rn(alpha, xc), __fmul_rn(beta, y[t]));
            continue;
        }
        const float kc = kap[t];
        float acc = 0.0f;
        const int nbr[6] = {t - nn, t + nn, t - n, t + n, t - 1, t + 1};
        const bool in[6] = {i > 0, i < n - 1, j > 0, j < n - 1, k > 0, k < n - 1};
#pragma unroll
        for (int s = 0; s < 6; ++s) {
            if (!in[s]) continue;
            const int nb = nbr[s];
            const float kf = face_kappa(kc, kap[nb]);
            acc = __fadd_rn(acc, (fl[nb] & 1) ? __fmul_rn(kf, xc) : __fmul_rn(kf, __fsub_rn(xc, x[nb])));
        }
        out[t] = __fadd_rn(__fmul_rn(alpha, __fadd_rn(xc, __fmul_rn(c_dt, acc))), __fmul_rn(beta, y[t]));
    }
}

}  // namespace hf
