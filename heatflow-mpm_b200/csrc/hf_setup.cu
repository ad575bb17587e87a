// hf_setup.cu -- scene set-up on the device: heater voxelisation, walls, the static sphere, and the mesh inside test.
//
// The reference builds a scene's statics on the host with numpy (heater.py:33-65 Heater.masks; solver.py:48-56 walls
// and the fixed-cell priority) and fills a mesh with particles through a Warp winding-number query (shapes.py:13-44).
// Here both run as kernels, so admitting a scene costs a few microseconds of GPU time and no host-to-device upload of
// its masks and face weights.
//
// Heater cells are classified in binary64 exactly as numpy evaluates heater.py:35-49:
//   * the frame coordinates s, q, r of a cell centre are the matmul `P @ a` of heater.py:38; numpy hands it to
//     OpenBLAS's dgemv, whose kernel on x86-64 hosts forms fma(p2, a2, fma(p0, a0, p1 * a1)) -- reproduced below with
//     explicit __fma_rn / __dmul_rn (the library is built with -fmad=false, so nothing else is contracted);
//   * np.hypot is the C library's hypot, which computes Borges' corrected square root ("An Improved Algorithm for
//     hypot(a,b)", C. F. Borges, 2019: h = sqrt(x^2 + y^2), then one correction step from the exact residual, evaluated
//     without fused operations) -- restated in hypot_corrected;
//   * every other operation is elementwise, one rounding each, in heater.py's order; the thresholds are evaluated on
//     the host from heater.py's own expressions and passed in.
// Because another host CPU may select a different dgemv kernel, the classifier also counts the cells whose class
// depends on a comparison closer than 1e-12 m to its threshold ("ambiguous"): with none, every faithful evaluation of
// heater.py gives the same classes.
#include <cmath>

#include "hf_device.cuh"
#include "hf_kernels.cuh"

namespace hf {

namespace {

constexpr double kAmbiguity = 1e-12;   // metres: comparisons closer than this to their threshold are reported

// Borges' hypot: sqrt of the sum of squares, corrected once by the residual of x^2 + y^2 - h^2 written as a sum of
// terms exact enough in binary64 (the two cases split on h <= 2 |y|), all operations rounded separately.
__device__ __forceinline__ double hypot_corrected(double x, double y) {
    double ax = fabs(x), ay = fabs(y);
    if (ax < ay) {
        const double t = ax;
        ax = ay;
        ay = t;
    }
    double h = __dsqrt_rn(__dadd_rn(__dmul_rn(ax, ax), __dmul_rn(ay, ay)));
    double t1, t2;
    if (h <= __dmul_rn(2.0, ay)) {
        const double delta = __dsub_rn(h, ay);
        t1 = __dmul_rn(ax, __dsub_rn(__dmul_rn(2.0, delta), ax));
        t2 = __dmul_rn(__dsub_rn(delta, __dmul_rn(2.0, __dsub_rn(ax, ay))), delta);
    } else {
        const double delta = __dsub_rn(h, ax);
        t1 = __dmul_rn(__dmul_rn(2.0, delta), __dsub_rn(ax, __dmul_rn(2.0, ay)));
        t2 = __dadd_rn(__dmul_rn(__dsub_rn(__dmul_rn(4.0, delta), ay), ay), __dmul_rn(delta, delta));
    }
    return __dsub_rn(h, __ddiv_rn(__dadd_rn(t1, t2), __dmul_rn(2.0, h)));
}

// heater.py:38 `P @ v` for one cell: OpenBLAS dgemv's evaluation order (see the file comment)
__device__ __forceinline__ double frame_dot(double p0, double p1, double p2, const double* v) {
    return __fma_rn(p2, v[2], __fma_rn(p0, v[0], __dmul_rn(p1, v[1])));
}

struct Margin {
    double m = 1e300;
    __device__ __forceinline__ void see(double v, double t) { m = fmin(m, fabs(__dsub_rn(v, t))); }
};

// heater.py:35-49: the class of cell (i, j, k) of the trough heater (0 air, 1 shell, 2 rod, 3 fan, 4 trough air)
__device__ int trough_class(const hf_heater_geometry& G, int i, int j, int k, double h, Margin& mg) {
    const double p0 = __dsub_rn(__dmul_rn((double)i + 0.5, h), G.centre[0]);
    const double p1 = __dsub_rn(__dmul_rn((double)j + 0.5, h), G.centre[1]);
    const double p2 = __dsub_rn(__dmul_rn((double)k + 0.5, h), G.centre[2]);
    const double s = frame_dot(p0, p1, p2, G.axis), q = frame_dot(p0, p1, p2, G.facing),
                 r = frame_dot(p0, p1, p2, G.up);
    const double rho = hypot_corrected(q, r), as = fabs(s);
    const double cap = fabs(__dsub_rn(as, G.half_length));
    const double rod_lo = hypot_corrected(__dadd_rn(q, G.rod_front), __dsub_rn(r, -G.rod_dz));
    const double rod_hi = hypot_corrected(__dadd_rn(q, G.rod_front), __dsub_rn(r, G.rod_dz));
    mg.see(as, G.half_length);
    mg.see(as, G.rod_half);
    mg.see(as, G.trough_half);
    mg.see(cap, G.cap_half);
    mg.see(q, 0.0);
    mg.see(rho, G.shell_in);
    mg.see(rho, G.shell_out);
    mg.see(rho, G.cap_radius);
    mg.see(rho, G.trough_radius);
    mg.see(rod_lo, G.rod_radius);
    mg.see(rod_hi, G.rod_radius);
    const bool behind = q <= 0.0;
    int c = 0;
    if (as <= G.half_length && behind && rho >= G.shell_in && rho <= G.shell_out) c = 1;   // reflector shell
    if (cap <= G.cap_half && behind && rho <= G.cap_radius) c = 1;                           // end caps
    const bool rod_span = as <= G.rod_half;
    if (rod_span && (rod_lo <= G.rod_radius || rod_hi <= G.rod_radius)) c = 2;               // the two rods
    if (G.fan) {
        mg.see(as, G.fan_half);
        mg.see(fabs(r), G.fan_high);
        mg.see(q, G.fan_depth);
        if (c == 0 && as <= G.fan_half && fabs(r) <= G.fan_high && q > 0.0 && q <= G.fan_depth) c = 3;
    }
    if (c == 0 && as <= G.trough_half && rho <= G.trough_radius && behind) c = 4;
    return c;
}

// The box heater: rods in [lo, hi) x [lo, hi) x [0, k_rod), trough air at k = k_rod, the fan layer above it.
__device__ __forceinline__ int box_class(const hf_heater_geometry& G, int i, int j, int k) {
    if (i < G.box_lo[0] || i >= G.box_hi[0] || j < G.box_lo[1] || j >= G.box_hi[1]) return 0;
    if (k < G.box_hi[2]) return 2;
    if (k == G.box_trough) return 4;
    if (G.fan && k == G.box_trough + 1) return 3;
    return 0;
}

__device__ __forceinline__ bool in_sphere(const hf_heater_geometry& G, int i, int j, int k, double h) {
    if (!G.sphere || i < G.sphere_lo || i >= G.sphere_hi || j < G.sphere_lo || j >= G.sphere_hi || k >= G.sphere_top)
        return false;
    const double dx = __dsub_rn(__dmul_rn((double)i + 0.5, h), G.sphere_c);
    const double dy = __dsub_rn(__dmul_rn((double)j + 0.5, h), G.sphere_c);
    const double dz = __dsub_rn(__dmul_rn((double)k + 0.5, h), G.sphere_zc);
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)) <= G.sphere_rr;
}

__device__ __forceinline__ int warp_count(bool b) { return __popc(__ballot_sync(0xffffffffu, b)); }

// One thread per cell: class byte (heater class | 8 for a sphere cell), flags (bit0 fixed, bit1 source), Dirichlet
// values and the static solid fraction.  Fixed cells: rods at t_rod, the side walls and the ceiling at t_amb (the floor
// is adiabatic), rods before walls (solver.py:48-53); sphere cells fixed at the sphere's temperature before both.
__global__ void __launch_bounds__(kThreads) k_heater_cells(hf_heater_geometry G, int n, double h, uint8_t* cls,
                                                           uint8_t* flags, float* tfix, float* alpha, int* counts) {
    const long long N = (long long)n * n * n;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long rounds = (N + stride - 1) / stride;   // every lane takes the same number of trips (warp ballots)
    const long long t0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    int sources = 0, ambiguous = 0;
    for (long long r = 0; r < rounds; ++r) {
        const long long t = t0 + r * stride;
        bool src = false, amb = false;
        if (t < N) {
            const int k = (int)(t % n), ij = (int)(t / n), j = ij % n, i = ij / n;
            int c = 0;
            if (G.kind == 1) {
                Margin mg;
                c = trough_class(G, i, j, k, h, mg);
                amb = mg.m <= kAmbiguity;
            } else if (G.kind == 2) {
                c = box_class(G, i, j, k);
            }
            const bool ball = in_sphere(G, i, j, k, h);
            const bool rod = c == 2, wall = i == 0 || i == n - 1 || j == 0 || j == n - 1 || k == n - 1;
            src = c == 3 || c == 4;
            const bool fixed = rod || wall || ball;
            float tf = rod ? __double2float_rn(G.t_rod) : (wall ? __double2float_rn(G.t_amb) : 0.0f);
            if (ball) tf = G.sphere_t;
            cls[t] = (uint8_t)(c | (ball ? 8 : 0));
            flags[t] = (uint8_t)((fixed ? 1 : 0) | (src ? 2 : 0));
            tfix[t] = tf;
            alpha[t] = (c == 1 || c == 2 || ball) ? 1.0f : 0.0f;
        }
        sources += warp_count(src);
        ambiguous += warp_count(amb);
    }
    if ((threadIdx.x & 31) == 0 && (sources || ambiguous)) {
        atomicAdd(counts + 0, sources);
        atomicAdd(counts + 1, ambiguous);
    }
}

// heater.py:53-63 on the three face lattices (the domain's outside counts as air): a face next to a solid cell (shell,
// rod or sphere) relaxes with K_SOLID toward rest, a face next to a fan cell and no solid one with K_FAN toward the fan
// velocity; momentum weights are K_FAN * fan * facing[axis], zero next to the sphere.
__global__ void __launch_bounds__(kThreads) k_heater_faces(hf_heater_geometry G, int n, const uint8_t* __restrict__ cls,
                                                           float* kx, float* ky, float* kz, float* mx, float* my,
                                                           float* mz) {
    const long long F = (long long)(n + 1) * n * n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 3 * F;
         t += (long long)gridDim.x * blockDim.x) {
        const int axis = (int)(t / F);
        const long long f = t - axis * F;
        int i, j, k, lo_ok, hi_ok;
        long long lo, hi;   // the two neighbouring cells
        if (axis == 0) {    // (n+1, n, n)
            k = (int)(f % n);
            j = (int)((f / n) % n);
            i = (int)(f / ((long long)n * n));
            lo = ((long long)(i - 1) * n + j) * n + k;
            hi = ((long long)i * n + j) * n + k;
            lo_ok = i > 0;
            hi_ok = i < n;
        } else if (axis == 1) {   // (n, n+1, n)
            k = (int)(f % n);
            j = (int)((f / n) % (n + 1));
            i = (int)(f / ((long long)(n + 1) * n));
            lo = ((long long)i * n + (j - 1)) * n + k;
            hi = ((long long)i * n + j) * n + k;
            lo_ok = j > 0;
            hi_ok = j < n;
        } else {                  // (n, n, n+1)
            k = (int)(f % (n + 1));
            j = (int)((f / (n + 1)) % n);
            i = (int)(f / ((long long)(n + 1) * n));
            lo = ((long long)i * n + j) * n + (k - 1);
            hi = ((long long)i * n + j) * n + k;
            lo_ok = k > 0;
            hi_ok = k < n;
        }
        const int a = lo_ok ? cls[lo] : 0, b = hi_ok ? cls[hi] : 0;
        const int ca = a & 7, cb = b & 7;
        const bool solid = ca == 1 || ca == 2 || cb == 1 || cb == 2;
        const bool fan = !solid && (ca == 3 || cb == 3);
        const bool ball = (a | b) & 8;
        float kv = solid ? G.k_solid : (fan ? G.k_fan : 0.0f);
        float mv = fan ? G.m_face[axis] : 0.0f;
        if (ball) {
            kv = G.k_solid;
            mv = 0.0f;
        }
        float* K = axis == 0 ? kx : (axis == 1 ? ky : kz);
        float* M = axis == 0 ? mx : (axis == 1 ? my : mz);
        K[f] = kv;
        M[f] = mv;
    }
}

// shapes.py:13-17 _inside: generalized winding number of every point against a triangle soup (Jacobson, Kavan and
// Sorkine-Hornung, "Robust Inside-Outside Segmentation using Generalized Winding Numbers", 2013): the sum of the
// triangles' signed solid angles over 4 pi, each by van Oosterom and Strackee's formula
// tan(Omega / 2) = a.(b x c) / (|a||b||c| + (a.b)|c| + (b.c)|a| + (c.a)|b|).  Blocks stage kWindTile triangles at a
// time in shared memory; every thread sums one point's angles in triangle order (deterministic).
constexpr int kWindTile = 256;

__global__ void __launch_bounds__(kThreads) k_winding(const float* __restrict__ tri, int num_tri,
                                                      const float* __restrict__ pts, int num_pts, float threshold,
                                                      int* __restrict__ flag, float* __restrict__ winding) {
    __shared__ float T[kWindTile * 9];
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = p < num_pts;
    const float px = live ? pts[3 * p] : 0.0f, py = live ? pts[3 * p + 1] : 0.0f, pz = live ? pts[3 * p + 2] : 0.0f;
    double sum = 0.0;
    for (int base = 0; base < num_tri; base += kWindTile) {
        const int m = min(kWindTile, num_tri - base);
        __syncthreads();
        for (int e = threadIdx.x; e < 9 * m; e += blockDim.x) T[e] = tri[9 * (long long)base + e];
        __syncthreads();
        float part = 0.0f;
        for (int t = 0; t < m; ++t) {
            const float* v = T + 9 * t;
            const float ax = v[0] - px, ay = v[1] - py, az = v[2] - pz;
            const float bx = v[3] - px, by = v[4] - py, bz = v[5] - pz;
            const float cx = v[6] - px, cy = v[7] - py, cz = v[8] - pz;
            const float la = sqrtf(ax * ax + ay * ay + az * az), lb = sqrtf(bx * bx + by * by + bz * bz),
                        lc = sqrtf(cx * cx + cy * cy + cz * cz);
            const float det = ax * (by * cz - bz * cy) + ay * (bz * cx - bx * cz) + az * (bx * cy - by * cx);
            const float den = la * lb * lc + (ax * bx + ay * by + az * bz) * lc + (bx * cx + by * cy + bz * cz) * la +
                              (cx * ax + cy * ay + cz * az) * lb;
            part += atan2f(det, den);
        }
        sum += (double)part;
    }
    if (live) {
        const float w = (float)(sum * (2.0 / (4.0 * 3.14159265358979323846)));
        flag[p] = w > threshold ? 1 : 0;
        if (winding) winding[p] = w;
    }
}

int grid_for(long long work) {
    long long b = (work + kThreads - 1) / kThreads;
    return (int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

}  // namespace

}  // namespace hf

extern "C" int hf_scene_statics(const hf_heater_geometry* geo, int n, double h, uint8_t* cell_class,
                                uint8_t* cell_flags, float* tfix, float* alpha, float* kx, float* ky, float* kz,
                                float* mx, float* my, float* mz, int32_t* counts, void* stream) {
    if (!geo || n < 2 || n > 1024 || !(h > 0.0) || !cell_class || !cell_flags || !tfix || !alpha || !kx || !ky ||
        !kz || !mx || !my || !mz || !counts)
        return hf::set_error(HF_ERR_ARG, "hf_scene_statics: null output, n outside [2, 1024] or h <= 0");
    if (geo->kind < 0 || geo->kind > 2)
        return hf::set_error(HF_ERR_ARG, "hf_scene_statics: heater kind must be 0 (none), 1 (trough) or 2 (box)");
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(counts, 0, 2 * sizeof(int32_t), st) != cudaSuccess)
        return hf::set_error(HF_ERR_CUDA, "hf_scene_statics: clearing the counters failed");
    const long long N = (long long)n * n * n, F = (long long)(n + 1) * n * n;
    hf::k_heater_cells<<<hf::grid_for(N), hf::kThreads, 0, st>>>(*geo, n, h, cell_class, cell_flags, tfix, alpha,
                                                                  counts);
    hf::k_heater_faces<<<hf::grid_for(3 * F), hf::kThreads, 0, st>>>(*geo, n, cell_class, kx, ky, kz, mx, my, mz);
    if (cudaGetLastError() != cudaSuccess) return hf::set_error(HF_ERR_CUDA, "hf_scene_statics: launch failed");
    return HF_OK;
}

extern "C" int hf_winding_inside(const float* tri, int num_tri, const float* points, int num_points, float threshold,
                                 int32_t* flag, float* winding, void* stream) {
    if (num_tri < 0 || num_points < 0 || (num_tri > 0 && !tri) || (num_points > 0 && (!points || !flag)))
        return hf::set_error(HF_ERR_ARG, "hf_winding_inside: null buffer or negative count");
    if (num_points == 0) return HF_OK;
    const int blocks = (num_points + hf::kThreads - 1) / hf::kThreads;
    hf::k_winding<<<blocks, hf::kThreads, 0, static_cast<cudaStream_t>(stream)>>>(tri, num_tri, points, num_points,
                                                                                   threshold, flag, winding);
    if (cudaGetLastError() != cudaSuccess) return hf::set_error(HF_ERR_CUDA, "hf_winding_inside: launch failed");
    return HF_OK;
}
