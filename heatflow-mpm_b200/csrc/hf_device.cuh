// hf_device.cuh -- device-side helpers shared by the kernels of libheatflow_b200.so.
//
// Arithmetic contract: every binary32 expression below is evaluated in the order the reference's Warp kernels state
// it, with one rounding per operation.  The library is compiled with -fmad=false so that nvcc does not contract a
// multiply and an add into an FMA; divisions are IEEE round-to-nearest (-prec-div=true, the default).  That makes the
// stencil, sampling and pointwise stages bit-identical to a serial binary32 evaluation of the same formulas.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/heatflow_b200.h"

namespace hf {

constexpr int kChunk = 1024;      // cells per work item
constexpr int kThreads = 256;     // threads per block of every chunked kernel
constexpr int kCellsPerThread = kChunk / kThreads;
// Blocks per chunk of the gather-bound stages (advection of T, the face stage): one cell per thread, so that a
// 96^3 scene's 864 chunks make 3456 blocks -- several waves of the 4 resident blocks per SM instead of 1.5, whose
// second, part-filled wave left most SMs idle.
constexpr int kStageSplit = 4;
static_assert(kCellsPerThread % kStageSplit == 0, "a chunk splits into whole cells per thread");
constexpr double kFxScale = 1099511627776.0;   // 2^40: particle fixed-point scale
constexpr double kFxInv = 1.0 / 1099511627776.0;
constexpr int kMaxScenes = 1024;

struct WorkItem {
    int scene;
    int first;   // first cell (linear index) of the chunk
};

// CG work item: a 4 x 8 x 32-cell tile (i, j, k) of one scene
constexpr int kTI = 4, kTJ = 8, kTK = 32;
struct TileItem {
    int scene, i0, j0, k0;
};

// ------------------------------------------------------------------------------------------ lattice arithmetic
__device__ __forceinline__ int clampi(int i, int lo, int hi) { return i < lo ? lo : (i > hi ? hi : i); }
__device__ __forceinline__ float minf_(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float maxf_(float a, float b) { return a > b ? a : b; }
// Warp's clamp(x, lo, hi) = min(max(lo, x), hi)
__device__ __forceinline__ float clampf_(float x, float lo, float hi) { return minf_(maxf_(lo, x), hi); }

// ---------------------------------------------------------------------------- division by a divisor known in advance
// Correctly rounded x / y when y is fixed for a whole kernel (the cell size h, or h^2), after Brisebarre, Muller &
// Raina, "Accelerating correctly rounded floating-point division when the divisor is known in advance", IEEE Trans.
// Computers 53(8), 2004: with zh = RN(1/y) and zl = RN((1 - y zh) / y) (1 - y zh is exact with one FMA), the quotient
// q = RN(x zh + RN(x zl)) is within one ulp of x / y; one correction step in the manner of Markstein (IBM J. Res. Dev.
// 34(1), 1990), r = x - q y (exact with one FMA) and RN(q + r zh), rounds it correctly.  Zero, tiny, huge and
// non-finite x take the ordinary IEEE division, so the result equals __fdiv_rn(x, y) bit for bit for every x (checked
// against the IEEE division over dense sweeps of x for the cell sizes in use).
struct DivBy {
    float y, zh, zl;
};

__device__ __forceinline__ DivBy div_by(float y) {
    const float zh = __fdiv_rn(1.0f, y);
    return DivBy{y, zh, __fdiv_rn(__fmaf_rn(-y, zh, 1.0f), y)};
}

__device__ __forceinline__ float div_rn(float x, const DivBy& d) {
    const float ax = fabsf(x);
    if (!(ax >= 0x1p-96f && ax <= 0x1p96f)) return __fdiv_rn(x, d.y);
    const float q = __fmaf_rn(x, d.zh, __fmul_rn(x, d.zl));
    return __fmaf_rn(__fmaf_rn(-q, d.y, x), d.zh, q);
}

// A sample point in grid units: each coordinate divided by h once (fields.py:14-15 divides before the offset), shared
// by every lattice sampled at that point.
struct GridPos {
    float x, y, z;
};

__device__ __forceinline__ GridPos grid_pos(float px, float py, float pz, const DivBy& h) {
    return GridPos{div_rn(px, h), div_rn(py, h), div_rn(pz, h)};
}

// fields.py:5-36 -- trilinear sample of an (nx,ny,nz) lattice with nodes at (i + off) h, indices clamped.
__device__ __forceinline__ float sample_at(const float* __restrict__ a, GridPos q, float ox, float oy, float oz, int nx,
                                           int ny, int nz) {
    float gx = __fsub_rn(q.x, ox);
    float gy = __fsub_rn(q.y, oy);
    float gz = __fsub_rn(q.z, oz);
    int ix = (int)floorf(gx), iy = (int)floorf(gy), iz = (int)floorf(gz);
    float fx = __fsub_rn(gx, (float)ix), fy = __fsub_rn(gy, (float)iy), fz = __fsub_rn(gz, (float)iz);
    float wx0 = __fsub_rn(1.0f, fx), wy0 = __fsub_rn(1.0f, fy), wz0 = __fsub_rn(1.0f, fz);
    int x0 = clampi(ix, 0, nx - 1), x1 = clampi(ix + 1, 0, nx - 1);
    int y0 = clampi(iy, 0, ny - 1), y1 = clampi(iy + 1, 0, ny - 1);
    int z0 = clampi(iz, 0, nz - 1), z1 = clampi(iz + 1, 0, nz - 1);
    const int sy = nz, sx = ny * nz;
    float s = 0.0f;
    // accumulation order dx, dy, dz with weight ((wx * wy) * wz) * a, as fields.py:29-35
    s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fmul_rn(wx0, wy0), wz0), __ldg(a + x0 * sx + y0 * sy + z0)));
    s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fmul_rn(wx0, wy0), fz), __ldg(a + x0 * sx + y0 * sy + z1)));
    s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fmul_rn(wx0, fy), wz0), __ldg(a + x0 * sx + y1 * sy + z0)));
    s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fmul_rn(wx0, fy), fz), __ldg(a + x0 * sx + y1 * sy + z1)));
    s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fmul_rn(fx, wy0), wz0), __ldg(a + x1 * sx + y0 * sy + z0)));
    s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fmul_rn(fx, wy0), fz), __ldg(a + x1 * sx + y0 * sy + z1)));
    s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fmul_rn(fx, fy), wz0), __ldg(a + x1 * sx + y1 * sy + z0)));
    s = __fadd_rn(s, __fmul_rn(__fmul_rn(__fmul_rn(fx, fy), fz), __ldg(a + x1 * sx + y1 * sy + z1)));
    return s;
}

// heat.py:50-52 -- harmonic face diffusivity; symmetric bit for bit in (a, b) because 2*a is exact
__device__ __forceinline__ float face_kappa(float a, float b) {
    return __fdiv_rn(__fmul_rn(__fmul_rn(2.0f, a), b), __fadd_rn(__fadd_rn(a, b), 1.0e-12f));
}

// linear cell index -> (i, j, k)
__device__ __forceinline__ void cell_ijk(int t, int n, int& i, int& j, int& k) {
    k = t % n;
    int q = t / n;
    j = q % n;
    i = q / n;
}

__device__ __forceinline__ float fx_to_float(long long v) { return __double2float_rn(__ll2double_rn(v) * kFxInv); }

// ------------------------------------------------------------------------------------------- memory ordering
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long global_timer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

}  // namespace hf
