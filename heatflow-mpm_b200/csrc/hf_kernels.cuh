// hf_kernels.cuh -- workspace layout and kernel declarations shared by the kernel files and the host API.
#pragma once

#include <cuda.h>

#include "hf_device.cuh"

namespace hf {

constexpr int kMaxLanes = 8;      // lanes of one streaming CG launch
constexpr int kGroupScenes = 32;  // scenes of one CG group (every block of a lane keeps all their scalars)
constexpr int kMaxGroups = 1024;  // groups of one launch (a kernel parameter: 16 KB)
constexpr int kMapsPerScene = 12; // TMA descriptors per scene in the workspace

// Scene groups of a streaming CG launch: group q = scenes [g[q].x, g[q].y), tiles [g[q].z, g[q].w).
struct GroupTable {
    int count, lanes;
    int4 g[kMaxGroups];
};

// Device pointers into the caller's workspace buffer (see hf_api.cu: workspace_layout).
struct Workspace {
    unsigned* bar;          // [2 kMaxLanes] barrier counters: heat lanes, then pressure lanes (reset every launch)
    unsigned* queue;        // [2] next group to solve (heat, pressure)
    int* lane_next;         // [2 kMaxLanes] group a lane works on
    int* err;               // [1] barrier timeout flag
    int* chunk_begin;       // [S+1] first chunk of every scene in the chunk table
    int* tile_begin;        // [S+1] first tile of every scene in the tile table
    const CUtensorMap* maps;  // [kMapsPerScene S] per scene: the stencil boxes z, p_0, p_1, alpha_f x, alpha_f y (cells),
                              // alpha_f z (cells); then tile boxes of x (p), p_0, p_1, r, Ap, D
    double* partA;          // [3 T] per-tile fp64 partials of CG phase A, component-major: component c of tile t at
                            // c * tiles + t (the single-reduction kernel: 5 components per 256-thread group)
    double* partB;          // [3 T] per-tile fp64 partials of the CG set-up and phase B (same layout)
    double* mean_part;      // [C] per-chunk fp64 sums of the pressure rhs
    int tiles;              // T: tiles of the plan, the component stride of partA / partB
};

// TMA descriptors of the tiled pressure stencil (resident CG): z, both search-direction buffers, alpha_f x (the u
// lattice), and the cell-layout copies of alpha_f y and z.
struct TileMaps {
    CUtensorMap z, p0, p1, ax, ayc, azc;      // pressure (and the z / p boxes of the heat system)
    CUtensorMap hkx, hky, hkzc, flags;        // heat: face diffusivities and the cell flags (bytes)
    CUtensorMap t0, t1;                       // heat: both temperature buffers (x0 is the one the parity selects)
};

__global__ void k_scatter(const hf_scene* __restrict__ scenes, int s);
__global__ void k_obstacle(const hf_scene* __restrict__ scenes, const WorkItem* __restrict__ work, int all_scenes);
__global__ void k_coeff(const hf_scene* __restrict__ scenes, const WorkItem* __restrict__ work, int all_scenes);
// the per-substep rebuild of one coupled scene, over its footprint boxes only
__global__ void k_obstacle_box(const hf_scene* __restrict__ scenes, int s);
__global__ void k_coeff_box(const hf_scene* __restrict__ scenes, int s);
__global__ void k_prestage(const hf_scene* __restrict__ scenes, const WorkItem* __restrict__ work, double dt);
__global__ void k_particle_update(const hf_scene* __restrict__ scenes, int s);
__global__ void k_face_tile(const hf_scene* __restrict__ scenes, const TileItem* __restrict__ tiles, double dt);
size_t face_tile_smem();   // dynamic shared memory of k_face_tile (512-thread blocks)
__global__ void k_advect_T_tile(const hf_scene* __restrict__ scenes, const TileItem* __restrict__ tiles, double dt);
size_t advect_tile_smem();   // dynamic shared memory of k_advect_T_tile (512-thread blocks)
__global__ void k_divergence(const hf_scene* __restrict__ scenes, const WorkItem* __restrict__ work, double dt, Workspace ws);
__global__ void k_cell_velocity(const hf_scene* __restrict__ scenes, int s, float* __restrict__ out);
__global__ void k_divergence_max(const hf_scene* __restrict__ scenes, int s, unsigned* __restrict__ out_bits);
__global__ void k_speed_max(const hf_scene* __restrict__ scenes, int s, unsigned* __restrict__ out_bits);
__global__ void k_laplacian_plain(int n, float h, float alpha, float beta, const float* __restrict__ p,
                                  const float* __restrict__ ax, const float* __restrict__ ay, const float* __restrict__ az,
                                  const float* __restrict__ y, float* __restrict__ out);
__global__ void k_divide_by(int count, const float* __restrict__ x, float y, float* __restrict__ out);
__global__ void k_heat_matvec_plain(int n, float h, float dt, float alpha, float beta, const float* __restrict__ x,
                                    const float* __restrict__ kap, const uint8_t* __restrict__ fl,
                                    const float* __restrict__ y, float* __restrict__ out);
// persistent cooperative Jacobi-PCG kernel over the groups of a GroupTable (heat = heat system, else pressure system +
// projection + end of substep; tma: pressure stencil staged by TMA from the workspace's descriptors, every scene of
// the table with n % 4 == 0); arguments: (const hf_scene*, const TileItem*, double dt, Workspace, GroupTable); the
// grid is a multiple of the table's lanes
const void* pcg_kernel(bool heat, bool tma);
// dynamic shared memory of the streaming kernel (tma: one stencil slot per block, staged with TMA)
size_t pcg_stream_smem(bool tma);
// register-resident single-scene variant (MAXC tiles per 256-thread group: 1, 2 or 3; blockDim = 256 x groups);
// arguments: (const hf_scene*, const TileItem*, int tile_lo, int tile_hi, double dt, Workspace, TileMaps) -- the
// scene's tiles; the TileMaps is used when tma; dynamic shared memory pcg_resident_smem(...)
const void* pcg_resident_kernel(bool heat, int maxc, bool tma);
size_t pcg_resident_smem(int groups, int maxc, bool tma, bool heat);
// single-reduction register-resident pressure solve of one scene with n % 4 == 0 (one grid barrier per CG iteration;
// uses hdiag as scratch), the same arguments and thread layout as the TMA resident variant; dynamic shared memory
// pcg_one_smem(groups, maxc)
const void* pcg_one_kernel(int maxc);
size_t pcg_one_smem(int groups, int maxc);
// limit of the CG kernels' bounded waits on the current device and the block kept from the first grid barrier
// (-1: none); synchronous (constant memory)
int set_wait_limit(unsigned long long limit_ns, int absent_block);
// device addresses of the per-scene chunk and tile offset tables inside a plan's workspace
void plan_offset_tables(const hf_plan* p, int** chunk_begin, int** tile_begin);
// record `msg` as the text of hf_last_error() and return `code`
int set_error(int code, const char* msg);

}  // namespace hf
