// hf_api.cu -- host side of the C ABI declared in include/heatflow_b200.h.
//
// Stateless apart from a per-device cache of SM count and cooperative-launch occupancies.  No function allocates device
// memory; the workspace layout below carves the caller's buffer (barrier counters, offset tables, the scenes' TMA
// descriptors, the CG partial sums).
#include <algorithm>
#include <cstdio>
#include <cudaTypedefs.h>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "hf_device.cuh"
#include "hf_kernels.cuh"

namespace {

thread_local std::string g_err;

int fail(int code, const char* what, cudaError_t e = cudaSuccess) {
    char buf[512];
    if (e != cudaSuccess)
        std::snprintf(buf, sizeof buf, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
    else
        std::snprintf(buf, sizeof buf, "%s", what);
    g_err = buf;
    return code;
}

#define HF_CUDA(call, what)                                  \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return fail(HF_ERR_CUDA, what, e_); \
    } while (0)

struct DeviceInfo {
    int sms = 0;
    int coop = 0;
    int occ_heat = 0, occ_pressure = 0, occ_pressure_tma = 0;
    size_t smem_optin = 0;
    bool ready = false;
    // occupancy of each resident variant [heat][tiles per group][tma][groups] (-1: not queried yet; the query also
    // raises the kernel's dynamic shared-memory limit)
    int res_occ[2][4][2][5];
    int pipe_occ[4][5];   // the single-reduction pressure variant [tiles per group][groups] (-1: not queried yet)
};

constexpr int kResGroupsMax[4] = {0, 4, 3, 2};   // 256-thread groups per block of the resident variant, by MAXC

std::mutex g_mu;
DeviceInfo g_dev[64];

int device_info(DeviceInfo** out) {
    int dev = 0;
    HF_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64) return fail(HF_ERR_DEVICE, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    DeviceInfo& d = g_dev[dev];
    if (!d.ready) {
        int major = 0;
        HF_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev), "cudaDeviceGetAttribute");
        if (major != 10) return fail(HF_ERR_DEVICE, "libheatflow_b200 is built for sm_100a (B200); this device is not sm_100");
        HF_CUDA(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
        HF_CUDA(cudaDeviceGetAttribute(&d.coop, cudaDevAttrCooperativeLaunch, dev), "cudaDeviceGetAttribute");
        HF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.occ_heat, hf::pcg_kernel(true, false), hf::kThreads, 0),
                "occupancy");
        HF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.occ_pressure, hf::pcg_kernel(false, false), hf::kThreads, 0),
                "occupancy");
        HF_CUDA(cudaFuncSetAttribute(hf::pcg_kernel(false, true), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)hf::pcg_stream_smem(true)),
                "smem attribute (streaming CG)");
        HF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.occ_pressure_tma, hf::pcg_kernel(false, true), hf::kThreads,
                                                              hf::pcg_stream_smem(true)),
                "occupancy");
        HF_CUDA(cudaFuncSetAttribute(hf::k_face_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hf::face_tile_smem()),
                "smem attribute (face stage)");
        HF_CUDA(cudaFuncSetAttribute(hf::k_advect_T_tile, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)hf::advect_tile_smem()),
                "smem attribute (temperature stage)");
        int optin = 0;
        HF_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev), "cudaDeviceGetAttribute");
        d.smem_optin = (size_t)optin;
        if (!d.coop) return fail(HF_ERR_DEVICE, "device does not support cooperative launches");
        std::memset(d.res_occ, 0xff, sizeof d.res_occ);
        std::memset(d.pipe_occ, 0xff, sizeof d.pipe_occ);
        d.ready = true;
    }
    *out = &d;
    return HF_OK;
}

constexpr long long kGroupCells = 2400000;   // cells of one CG group by default (one 128^3 or two 96^3 scenes)
constexpr size_t kHeadBytes = 256;           // barrier counters, group queue, lane slots, timeout flag

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

struct Layout {
    size_t head, chunk_begin, tile_begin, maps, partA, partB, mean_part, total;
};

Layout layout(int S, int C, int T) {
    Layout L{};
    size_t o = 0;
    L.head = o;                      // bar[2 kMaxLanes], queue[2], lane_next[2 kMaxLanes], err -> 256 bytes
    o = align_up(o + kHeadBytes, 256);
    L.chunk_begin = o;
    o = align_up(o + sizeof(int) * (size_t)(S + 1), 256);
    L.tile_begin = o;
    o = align_up(o + sizeof(int) * (size_t)(S + 1), 256);
    L.maps = o;                      // kMapsPerScene TMA descriptors per scene (128 bytes each)
    o = align_up(o + sizeof(CUtensorMap) * hf::kMapsPerScene * (size_t)S, 256);
    L.partA = o;                     // 5 doubles per tile, component-major (3 components used by the classic variants)
    o = align_up(o + sizeof(double) * 5 * (size_t)T, 256);
    L.partB = o;
    o = align_up(o + sizeof(double) * 5 * (size_t)T, 256);
    L.mean_part = o;
    o = align_up(o + sizeof(double) * (size_t)C, 256);
    L.total = o;
    return L;
}

hf::Workspace workspace(const hf_plan* p) {
    const Layout L = layout(p->num_scenes, p->num_chunks, p->num_tiles);
    char* b = static_cast<char*>(p->workspace);
    hf::Workspace w;
    w.bar = reinterpret_cast<unsigned*>(b + L.head);
    w.queue = w.bar + 2 * hf::kMaxLanes;
    w.lane_next = reinterpret_cast<int*>(w.queue + 2);
    w.err = w.lane_next + 2 * hf::kMaxLanes;
    w.chunk_begin = reinterpret_cast<int*>(b + L.chunk_begin);
    w.tile_begin = reinterpret_cast<int*>(b + L.tile_begin);
    w.maps = reinterpret_cast<const CUtensorMap*>(b + L.maps);
    w.partA = reinterpret_cast<double*>(b + L.partA);
    w.partB = reinterpret_cast<double*>(b + L.partB);
    w.mean_part = reinterpret_cast<double*>(b + L.mean_part);
    w.tiles = p->num_tiles;
    return w;
}

int tiles_of(int n) { return ((n + hf::kTI - 1) / hf::kTI) * ((n + hf::kTJ - 1) / hf::kTJ) * ((n + hf::kTK - 1) / hf::kTK); }

// TMA descriptor of a 3-D float array (k fastest) of dims (nk, nj, ni) with a box (bk, bj, bi)
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

int encode_map(CUtensorMap* m, const float* base, int nk, int nj, int ni, int bk, int bj, int bi) {
    if (!g_encode) {
        cudaDriverEntryPointQueryResult q;
        HF_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", reinterpret_cast<void**>(&g_encode), cudaEnableDefault, &q),
                "cudaGetDriverEntryPoint(cuTensorMapEncodeTiled)");
        if (q != cudaDriverEntryPointSuccess || !g_encode) return fail(HF_ERR_DEVICE, "cuTensorMapEncodeTiled unavailable");
    }
    const cuuint64_t dims[3] = {(cuuint64_t)nk, (cuuint64_t)nj, (cuuint64_t)ni};
    const cuuint64_t strides[2] = {(cuuint64_t)nk * 4u, (cuuint64_t)nk * nj * 4u};
    const cuuint32_t box[3] = {(cuuint32_t)bk, (cuuint32_t)bj, (cuuint32_t)bi};
    const cuuint32_t es[3] = {1, 1, 1};
    CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, es,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(HF_ERR_DEVICE, "cuTensorMapEncodeTiled failed");
    return HF_OK;
}

// The six TMA descriptors of a scene's tiled pressure stencil (order of hf::TileMaps): z and both search-direction
// buffers with a one-cell halo, alpha_f x on its face lattice, alpha_f y and z in cell layout.
static_assert(sizeof(hf::TileMaps) == 12 * sizeof(CUtensorMap), "TileMaps is twelve consecutive descriptors");

// a 3-D byte array (k fastest) of dims (nk, nj, ni) with a box (bk, bj, bi): nk and bk multiples of 16
int encode_map_u8(CUtensorMap* m, const uint8_t* base, int nk, int nj, int ni, int bk, int bj, int bi) {
    if (!g_encode) {
        CUtensorMap probe;
        int rc = encode_map(&probe, reinterpret_cast<const float*>(base), 4, 1, 1, 4, 1, 1);   // loads the entry point
        if (rc) return rc;
    }
    const cuuint64_t dims[3] = {(cuuint64_t)nk, (cuuint64_t)nj, (cuuint64_t)ni};
    const cuuint64_t strides[2] = {(cuuint64_t)nk, (cuuint64_t)nk * nj};
    const cuuint32_t box[3] = {(cuuint32_t)bk, (cuuint32_t)bj, (cuuint32_t)bi};
    const cuuint32_t es[3] = {1, 1, 1};
    CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<uint8_t*>(base), dims, strides, box, es,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(HF_ERR_DEVICE, "cuTensorMapEncodeTiled (bytes) failed");
    return HF_OK;
}

// The TMA descriptors of a scene's tiled heat stencil: the z / p boxes of the pressure geometry, the face
// diffusivities x (face lattice, like alpha_f x), y (rows j0..j0+8 of the (n, n+1, n) face lattice) and z (cell-layout
// copy), and the cell flags with a one-cell halo (k origin 16-byte aligned).  Needs n % 16 == 0 (byte rows).
int encode_heat_maps(const hf_scene& sc, hf::TileMaps& m) {
    const int n = sc.n;
    int rc;
    if ((rc = encode_map(&m.z, sc.cg_z, n, n, n, 40, 10, 6))) return rc;
    if ((rc = encode_map(&m.p0, sc.cg_p[0], n, n, n, 40, 10, 6))) return rc;
    if ((rc = encode_map(&m.p1, sc.cg_p[1], n, n, n, 40, 10, 6))) return rc;
    if ((rc = encode_map(&m.hkx, sc.hkx, n, n, n + 1, 32, 8, 5))) return rc;
    if ((rc = encode_map(&m.hky, sc.hky, n, n + 1, n, 32, 9, 4))) return rc;
    if ((rc = encode_map(&m.hkzc, sc.hkzc, n, n, n, 36, 8, 4))) return rc;
    if ((rc = encode_map(&m.t0, sc.T[0], n, n, n, 40, 10, 6))) return rc;
    if ((rc = encode_map(&m.t1, sc.T[1], n, n, n, 40, 10, 6))) return rc;
    return encode_map_u8(&m.flags, sc.cell_flags, n, n, n, 64, 10, 6);
}

int encode_scene_maps(const hf_scene& sc, CUtensorMap* m) {
    const int n = sc.n;
    int rc;
    if ((rc = encode_map(&m[0], sc.cg_z, n, n, n, 40, 10, 6))) return rc;
    if ((rc = encode_map(&m[1], sc.cg_p[0], n, n, n, 40, 10, 6))) return rc;
    if ((rc = encode_map(&m[2], sc.cg_p[1], n, n, n, 40, 10, 6))) return rc;
    if ((rc = encode_map(&m[3], sc.ax, n, n, n + 1, 32, 8, 5))) return rc;
    if ((rc = encode_map(&m[4], sc.ayc, n, n, n, 32, 9, 4))) return rc;
    return encode_map(&m[5], sc.azc, n, n, n, 36, 8, 4);
}

int check_plan(const hf_plan* p) {
    if (!p || !p->scenes_host || !p->scenes_dev || !p->work_dev || !p->workspace) return fail(HF_ERR_ARG, "incomplete hf_plan");
    if (p->num_scenes <= 0 || p->num_scenes > hf::kMaxScenes) return fail(HF_ERR_ARG, "num_scenes out of range (1..1024)");
    if (!p->tiles_dev) return fail(HF_ERR_ARG, "incomplete hf_plan (tile table)");
    if (p->workspace_bytes < layout(p->num_scenes, p->num_chunks, p->num_tiles).total)
        return fail(HF_ERR_WORKSPACE, "workspace smaller than hf_workspace_bytes()");
    return HF_OK;
}

inline cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }

bool any_flag(const hf_plan* p, unsigned f) {
    for (int s = 0; s < p->num_scenes; ++s)
        if ((p->scenes_host[s].flags & HF_FLAG_ACTIVE) && (p->scenes_host[s].flags & f)) return true;
    return false;
}

// The resident variant for a plan with one active scene whose tiles fit one block per SM.  Returns HF_OK after
// launching, or -1 when the scene does not fit (the caller falls back to the streaming kernel).
int launch_resident(const hf_plan* p, DeviceInfo* d, bool heat, double dt, int s, void* stream) {
    hf::Workspace ws = workspace(p);
    const hf_scene* scenes = static_cast<const hf_scene*>(p->scenes_dev);
    const hf::TileItem* tiles = static_cast<const hf::TileItem*>(p->tiles_dev);
    const hf_scene& sc = p->scenes_host[s];
    int t_lo = 0, t_hi = p->num_tiles, rc;
    const int nt = t_hi - t_lo;
    const int G = nt < d->sms ? nt : d->sms;
    const int tpb = (nt + G - 1) / G;
    // TMA-staged stencils: pressure with n % 4 == 0 (16-byte float rows), heat with n % 16 == 0 (16-byte flag rows)
    const bool tma = !(p->options & HF_PLAN_NO_TMA) &&
                     (heat ? (sc.n % 16 == 0 && sc.hkzc && sc.hkx && sc.hky && sc.cell_flags) : (sc.n % 4 == 0));
    const int want = (int)((p->options >> HF_PLAN_RES_TILES_SHIFT) & 3u);   // 0: the first that fits
    // the single-reduction pressure solve (one grid barrier per iteration) when the plan asks for it, the stencil is
    // staged and its scratch vectors exist
    const bool pipe = !heat && tma && (p->options & HF_PLAN_SINGLE_REDUCTION_CG) && sc.cg_r && sc.cg_z && sc.cg_Ap &&
                      sc.hdiag && sc.pdiag && sc.cg_p[0] && sc.cg_p[1];
    // tiles per group: the fewest that fit; the single-reduction pressure kernel prefers three (two 256-thread groups
    // of 128 registers per thread: its per-thread state does not fit the 80 registers of a 768-thread block)
    const bool three_first = pipe && !want && tpb > 4;
    for (int mi = 0; mi < 3; ++mi) {
        const int m = want ? want + mi : (three_first ? 3 - mi : 1 + mi);
        if (m > 3) break;
        const int groups = (tpb + m - 1) / m;
        if (groups > kResGroupsMax[m]) continue;
        // the single-reduction kernel publishes one set of partials per 256-thread group into buffers sized by tiles
        if (pipe && G * groups > nt) continue;
        const void* fn = pipe ? hf::pcg_one_kernel(m) : hf::pcg_resident_kernel(heat, m, tma);
        const size_t smem = pipe ? hf::pcg_one_smem(groups, m) : hf::pcg_resident_smem(groups, m, tma, heat);
        if (smem > d->smem_optin) continue;
        int& occ = pipe ? d->pipe_occ[m][groups] : d->res_occ[heat][m][tma][groups];
        if (occ < 0) {
            if (smem > 48 * 1024)
                HF_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem attribute");
            int o = 0;
            HF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, fn, 256 * groups, smem), "occupancy (resident)");
            occ = o;
        }
        if (occ < 1) continue;
        hf::TileMaps maps;
        std::memset(&maps, 0, sizeof maps);
        if (tma && (rc = heat ? encode_heat_maps(sc, maps) : encode_scene_maps(sc, &maps.z))) return rc;
        HF_CUDA(cudaMemsetAsync(ws.bar, 0, kHeadBytes, S(stream)), "cudaMemsetAsync(barrier)");
        void* args[] = {(void*)&scenes, (void*)&tiles, (void*)&t_lo, (void*)&t_hi, (void*)&dt, (void*)&ws, (void*)&maps};
        HF_CUDA(cudaLaunchCooperativeKernel(fn, dim3(G), dim3(256 * groups), args, smem, S(stream)),
                "cooperative launch (resident CG)");
        return HF_OK;
    }
    return -1;
}

// Both CG solves of a plan.  One active scene: the resident variant where it fits.  Otherwise one launch of the
// streaming kernel: the active scenes are cut, in table order, into groups of at most kGroupScenes scenes and
// group_cells cells (default kGroupCells: a group's CG vectors stay in L2), solved by the lanes of the grid.
int launch_pcg(const hf_plan* p, bool heat, double dt, void* stream) {
    DeviceInfo* d = nullptr;
    int rc = device_info(&d);
    if (rc) return rc;
    if (p->num_tiles == 0) return HF_OK;
    int nactive = 0, last = -1, total = 0;
    bool correction = false;   // the outer defect correction runs in the streaming kernel only
    for (int s = 0; s < p->num_scenes; ++s)
        if (p->scenes_host[s].flags & HF_FLAG_ACTIVE) {
            ++nactive;
            last = s;
            total += tiles_of(p->scenes_host[s].n);
            correction = correction || (p->scenes_host[s].flags & HF_FLAG_DEFECT_CORRECTION);
        }
    if (total != p->num_tiles) return fail(HF_ERR_ARG, "plan changed since hf_plan_upload");
    if (nactive == 1 && !correction && !(p->options & HF_PLAN_STREAMING_CG) &&
        !(heat && (p->options & HF_PLAN_STREAMING_HEAT))) {
        rc = launch_resident(p, d, heat, dt, last, stream);
        if (rc != -1) return rc;
    }
    static thread_local hf::GroupTable gt;   // 16 KB: kept off the stack; the launch copies it
    gt.count = 0;
    const long long budget = p->group_cells > 0 ? p->group_cells : kGroupCells;
    int s_lo = -1, s_last = -1, t_lo = 0, t = 0;
    long long cells = 0;
    for (int s = 0; s <= p->num_scenes; ++s) {
        const bool end = s == p->num_scenes;
        if (!end && !(p->scenes_host[s].flags & HF_FLAG_ACTIVE)) continue;
        const long long c = end ? 0 : (long long)p->scenes_host[s].n * p->scenes_host[s].n * p->scenes_host[s].n;
        if (s_lo >= 0 && (end || cells + c > budget || s + 1 - s_lo > hf::kGroupScenes)) {
            // the group ends after its last active scene: [s_lo, s_last] spans at most kGroupScenes scenes
            if (gt.count == hf::kMaxGroups) return fail(HF_ERR_ARG, "more CG groups than one launch takes");
            gt.g[gt.count++] = make_int4(s_lo, s_last + 1, t_lo, t);
            s_lo = -1;
        }
        if (end) break;
        if (s_lo < 0) {
            s_lo = s;
            t_lo = t;
            cells = 0;
        }
        cells += c;
        s_last = s;
        t += tiles_of(p->scenes_host[s].n);
    }
    // the pressure stencil from TMA-staged boxes when the plan's descriptors exist and every active scene has them
    bool tma = !heat && (p->options & HF_PLAN_MAPS_READY) && !(p->options & HF_PLAN_NO_TMA);
    for (int s = 0; tma && s < p->num_scenes; ++s) {
        const hf_scene& sc = p->scenes_host[s];
        // the same test as hf_plan_upload's: only then does the workspace hold this scene's descriptors
        if ((sc.flags & HF_FLAG_ACTIVE) && (sc.n % 4 != 0 || !sc.cg_z || !sc.cg_p[0] || !sc.cg_p[1] || !sc.ax || !sc.ayc ||
                                            !sc.azc || !sc.p || !sc.cg_r || !sc.cg_Ap || !sc.pdiag))
            tma = false;
    }
    const int occ = heat ? d->occ_heat : tma ? d->occ_pressure_tma : d->occ_pressure;
    if (occ <= 0) return fail(HF_ERR_DEVICE, "persistent CG kernel does not fit on an SM");
    int lanes = (int)((p->options >> HF_PLAN_LANES_SHIFT) & 15u);
    if (lanes <= 0) lanes = 1;
    if (lanes > hf::kMaxLanes) lanes = hf::kMaxLanes;
    if (lanes > gt.count) lanes = gt.count;
    int grid = p->persistent_blocks > 0 ? p->persistent_blocks : d->sms * (occ < 2 ? occ : 2);
    if (grid > d->sms * occ) grid = d->sms * occ;
    grid -= grid % lanes;
    if (grid < lanes) grid = lanes;
    gt.lanes = lanes;
    hf::Workspace ws = workspace(p);
    const hf_scene* scenes = static_cast<const hf_scene*>(p->scenes_dev);
    const hf::TileItem* tiles = static_cast<const hf::TileItem*>(p->tiles_dev);
    HF_CUDA(cudaMemsetAsync(ws.bar, 0, kHeadBytes, S(stream)), "cudaMemsetAsync(barrier)");
    void* args[] = {(void*)&scenes, (void*)&tiles, (void*)&dt, (void*)&ws, (void*)&gt};
    HF_CUDA(cudaLaunchCooperativeKernel(hf::pcg_kernel(heat, tma), dim3(grid), dim3(hf::kThreads), args,
                                        hf::pcg_stream_smem(tma), S(stream)),
            "cooperative launch (CG)");
    return HF_OK;
}

}  // namespace

namespace hf {
int set_error(int code, const char* msg) { return fail(code, msg); }

void plan_offset_tables(const hf_plan* p, int** chunk_begin, int** tile_begin) {
    const Workspace w = workspace(p);
    *chunk_begin = w.chunk_begin;
    *tile_begin = w.tile_begin;
}
}  // namespace hf

extern "C" {

int hf_abi_version(void) { return HF_ABI_VERSION; }

const char* hf_last_error(void) { return g_err.c_str(); }

int hf_cells_per_chunk(void) { return hf::kChunk; }

int hf_chunks_for(int n) {
    if (n <= 0) return 0;
    const long long N = (long long)n * n * n;
    return (int)((N + hf::kChunk - 1) / hf::kChunk);
}

size_t hf_workspace_bytes(int num_scenes, int num_chunks, int num_tiles) {
    return layout(num_scenes, num_chunks, num_tiles).total;
}

int hf_tiles_for(int n) { return n > 0 ? tiles_of(n) : 0; }

int hf_plan_upload(hf_plan* p, void* stream) {
    if (!p || !p->scenes_host || !p->scenes_dev || !p->work_dev || !p->tiles_dev || !p->workspace)
        return fail(HF_ERR_ARG, "incomplete hf_plan");
    if (p->num_scenes <= 0 || p->num_scenes > hf::kMaxScenes) return fail(HF_ERR_ARG, "num_scenes out of range (1..1024)");
    std::vector<hf::WorkItem> work;
    std::vector<hf::TileItem> tiles;
    std::vector<int> begin(p->num_scenes + 1, 0), tbegin(p->num_scenes + 1, 0);
    for (int s = 0; s < p->num_scenes; ++s) {
        const hf_scene& sc = p->scenes_host[s];
        begin[s] = (int)work.size();
        tbegin[s] = (int)tiles.size();
        if (!(sc.flags & HF_FLAG_ACTIVE)) continue;
        if (sc.n < 2 || sc.n > 1024) return fail(HF_ERR_ARG, "scene edge n out of range (2..1024)");
        if (!sc.state) return fail(HF_ERR_ARG, "scene without a state block");
        const long long N = (long long)sc.n * sc.n * sc.n;
        for (long long f = 0; f < N; f += hf::kChunk) work.push_back(hf::WorkItem{s, (int)f});
        // k fastest, then i, then j: the six neighbours of a tile are at most (n / 32) (n / 4) tiles away in the
        // table, so tiles solved side by side share their halo rows in L2
        for (int j0 = 0; j0 < sc.n; j0 += hf::kTJ)
            for (int i0 = 0; i0 < sc.n; i0 += hf::kTI)
                for (int k0 = 0; k0 < sc.n; k0 += hf::kTK) tiles.push_back(hf::TileItem{s, i0, j0, k0});
    }
    begin[p->num_scenes] = (int)work.size();
    tbegin[p->num_scenes] = (int)tiles.size();
    p->num_chunks = (int)work.size();
    p->num_tiles = (int)tiles.size();
    const Layout L = layout(p->num_scenes, p->num_chunks, p->num_tiles);
    if (p->workspace_bytes < L.total) return fail(HF_ERR_WORKSPACE, "workspace smaller than hf_workspace_bytes()");
    HF_CUDA(cudaMemsetAsync(p->workspace, 0, L.total, S(stream)), "cudaMemsetAsync(workspace)");
    HF_CUDA(cudaMemcpyAsync(p->scenes_dev, p->scenes_host, sizeof(hf_scene) * p->num_scenes, cudaMemcpyHostToDevice, S(stream)),
            "upload scene table");
    if (!work.empty())
        HF_CUDA(cudaMemcpyAsync(p->work_dev, work.data(), sizeof(hf::WorkItem) * work.size(), cudaMemcpyHostToDevice, S(stream)),
                "upload chunk table");
    if (!tiles.empty())
        HF_CUDA(cudaMemcpyAsync(p->tiles_dev, tiles.data(), sizeof(hf::TileItem) * tiles.size(), cudaMemcpyHostToDevice, S(stream)),
                "upload tile table");
    char* b = static_cast<char*>(p->workspace);
    HF_CUDA(cudaMemcpyAsync(b + L.chunk_begin, begin.data(), sizeof(int) * begin.size(), cudaMemcpyHostToDevice, S(stream)),
            "upload chunk offsets");
    HF_CUDA(cudaMemcpyAsync(b + L.tile_begin, tbegin.data(), sizeof(int) * tbegin.size(), cudaMemcpyHostToDevice, S(stream)),
            "upload tile offsets");
    // TMA descriptors of every active scene whose stencil boxes fit the alignment rules (n % 4 == 0); zero otherwise
    std::vector<CUtensorMap> maps(hf::kMapsPerScene * (size_t)p->num_scenes);
    std::memset(maps.data(), 0, sizeof(CUtensorMap) * maps.size());
    for (int s = 0; s < p->num_scenes; ++s) {
        const hf_scene& sc = p->scenes_host[s];
        if (!(sc.flags & HF_FLAG_ACTIVE) || sc.n % 4 != 0 || !sc.cg_z || !sc.cg_p[0] || !sc.cg_p[1] || !sc.ax || !sc.ayc ||
            !sc.azc || !sc.p || !sc.cg_r || !sc.cg_Ap || !sc.pdiag)
            continue;
        CUtensorMap* m = &maps[hf::kMapsPerScene * (size_t)s];
        int rc = encode_scene_maps(sc, m);
        if (rc) return rc;
        // the CG vectors of the tile's own cells, one (32, 8, 4) box each: x (the pressure), p_0, p_1, r, Ap, D
        const float* own[6] = {sc.p, sc.cg_p[0], sc.cg_p[1], sc.cg_r, sc.cg_Ap, sc.pdiag};
        for (int q = 0; q < 6; ++q)
            if ((rc = encode_map(&m[6 + q], own[q], sc.n, sc.n, sc.n, 32, 8, 4))) return rc;
    }
    HF_CUDA(cudaMemcpyAsync(b + L.maps, maps.data(), sizeof(CUtensorMap) * maps.size(), cudaMemcpyHostToDevice, S(stream)),
            "upload TMA descriptors");
    HF_CUDA(cudaStreamSynchronize(S(stream)), "cudaStreamSynchronize(plan upload)");
    p->options |= HF_PLAN_MAPS_READY;
    return HF_OK;
}

int hf_obstacle_fields(const hf_plan* p, int all_scenes, void* stream) {
    int rc = check_plan(p);
    if (rc) return rc;
    const hf_scene* scenes = static_cast<const hf_scene*>(p->scenes_dev);
    const hf::WorkItem* work = static_cast<const hf::WorkItem*>(p->work_dev);
    const bool coupled = any_flag(p, HF_FLAG_PARTICLES);
    if (!coupled && !all_scenes) return HF_OK;
    for (int s = 0; s < p->num_scenes; ++s) {
        const hf_scene& sc = p->scenes_host[s];
        if (!(sc.flags & HF_FLAG_ACTIVE) || !(sc.flags & HF_FLAG_PARTICLES) || sc.n_particles <= 0) continue;
        if (!sc.acc || !sc.pos || !sc.pvel || !sc.ptemp) return fail(HF_ERR_ARG, "coupled scene without particle buffers");
        hf::k_scatter<<<(sc.n_particles + hf::kThreads - 1) / hf::kThreads, hf::kThreads, 0, S(stream)>>>(scenes, s);
    }
    if (!all_scenes) {
        // the substep's rebuild: each coupled scene over its footprint boxes only
        for (int s = 0; s < p->num_scenes; ++s) {
            const hf_scene& sc = p->scenes_host[s];
            if (!(sc.flags & HF_FLAG_ACTIVE) || !(sc.flags & HF_FLAG_PARTICLES) || sc.n_particles <= 0) continue;
            hf::k_obstacle_box<<<296, hf::kThreads, 0, S(stream)>>>(scenes, s);
        }
        for (int s = 0; s < p->num_scenes; ++s) {
            const hf_scene& sc = p->scenes_host[s];
            if (!(sc.flags & HF_FLAG_ACTIVE) || !(sc.flags & HF_FLAG_PARTICLES) || sc.n_particles <= 0) continue;
            hf::k_coeff_box<<<296, hf::kThreads, 0, S(stream)>>>(scenes, s);
        }
    } else if (p->num_chunks) {
        hf::k_obstacle<<<p->num_chunks, hf::kThreads, 0, S(stream)>>>(scenes, work, all_scenes);
        hf::k_coeff<<<p->num_chunks, hf::kThreads, 0, S(stream)>>>(scenes, work, all_scenes);
    }
    HF_CUDA(cudaGetLastError(), "launch (obstacle fields)");
    return HF_OK;
}

int hf_temperature_stage(const hf_plan* p, double dt, void* stream) {
    int rc = check_plan(p);
    if (rc) return rc;
    if (!p->num_chunks) return HF_OK;
    const hf_scene* scenes = static_cast<const hf_scene*>(p->scenes_dev);
    const hf::WorkItem* work = static_cast<const hf::WorkItem*>(p->work_dev);
    DeviceInfo* d = nullptr;
    if ((rc = device_info(&d))) return rc;
    hf::k_prestage<<<p->num_chunks, hf::kThreads, 0, S(stream)>>>(scenes, work, dt);
    // one 512-thread block per CG tile, the old velocities and Tw around the tile staged in shared memory
    hf::k_advect_T_tile<<<p->num_tiles, 512, hf::advect_tile_smem(), S(stream)>>>(
        scenes, static_cast<const hf::TileItem*>(p->tiles_dev), dt);
    HF_CUDA(cudaGetLastError(), "launch (temperature stage)");
    return HF_OK;
}

int hf_heat_solve(const hf_plan* p, double dt, void* stream) {
    int rc = check_plan(p);
    if (rc) return rc;
    return launch_pcg(p, true, dt, stream);
}

int hf_particle_update(const hf_plan* p, void* stream) {
    int rc = check_plan(p);
    if (rc) return rc;
    const hf_scene* scenes = static_cast<const hf_scene*>(p->scenes_dev);
    for (int s = 0; s < p->num_scenes; ++s) {
        const hf_scene& sc = p->scenes_host[s];
        if (!(sc.flags & HF_FLAG_ACTIVE) || !(sc.flags & HF_FLAG_PARTICLES) || sc.n_particles <= 0) continue;
        hf::k_particle_update<<<(sc.n_particles + hf::kThreads - 1) / hf::kThreads, hf::kThreads, 0, S(stream)>>>(scenes, s);
    }
    HF_CUDA(cudaGetLastError(), "launch (particle update)");
    return HF_OK;
}

int hf_face_stage(const hf_plan* p, double dt, void* stream) {
    int rc = check_plan(p);
    if (rc) return rc;
    if (!p->num_tiles) return HF_OK;
    DeviceInfo* d = nullptr;
    if ((rc = device_info(&d))) return rc;
    // one 512-thread block per CG tile, the old velocities around the tile staged in shared memory
    hf::k_face_tile<<<p->num_tiles, 512, hf::face_tile_smem(), S(stream)>>>(static_cast<const hf_scene*>(p->scenes_dev),
                                                                        static_cast<const hf::TileItem*>(p->tiles_dev), dt);
    HF_CUDA(cudaGetLastError(), "launch (face stage)");
    return HF_OK;
}

int hf_divergence_stage(const hf_plan* p, double dt, void* stream) {
    int rc = check_plan(p);
    if (rc) return rc;
    if (!p->num_chunks) return HF_OK;
    hf::k_divergence<<<p->num_chunks, hf::kChunk, 0, S(stream)>>>(static_cast<const hf_scene*>(p->scenes_dev),
                                                                   static_cast<const hf::WorkItem*>(p->work_dev), dt,
                                                                   workspace(p));
    HF_CUDA(cudaGetLastError(), "launch (divergence)");
    return HF_OK;
}

int hf_pressure_cg(const hf_plan* p, double dt, void* stream) {
    int rc = check_plan(p);
    if (rc) return rc;
    return launch_pcg(p, false, dt, stream);
}

int hf_pressure_solve(const hf_plan* p, double dt, void* stream) {
    int rc = hf_divergence_stage(p, dt, stream);
    if (rc) return rc;
    return hf_pressure_cg(p, dt, stream);
}

int hf_substep(const hf_plan* p, double dt, void* stream) {
    int rc;
    if ((rc = hf_obstacle_fields(p, 0, stream))) return rc;
    if ((rc = hf_temperature_stage(p, dt, stream))) return rc;
    if ((rc = hf_heat_solve(p, dt, stream))) return rc;
    if ((rc = hf_particle_update(p, stream))) return rc;
    if ((rc = hf_face_stage(p, dt, stream))) return rc;
    return hf_pressure_solve(p, dt, stream);
}

int hf_cell_velocity(const hf_plan* p, int s, float* out, void* stream) {
    int rc = check_plan(p);
    if (rc) return rc;
    if (s < 0 || s >= p->num_scenes || !out) return fail(HF_ERR_ARG, "bad scene index or output");
    hf::k_cell_velocity<<<592, 256, 0, S(stream)>>>(static_cast<const hf_scene*>(p->scenes_dev), s, out);
    HF_CUDA(cudaGetLastError(), "launch (cell velocity)");
    return HF_OK;
}

int hf_divergence_max(const hf_plan* p, int s, float* out_dev, void* stream) {
    int rc = check_plan(p);
    if (rc) return rc;
    if (s < 0 || s >= p->num_scenes || !out_dev) return fail(HF_ERR_ARG, "bad scene index or output");
    HF_CUDA(cudaMemsetAsync(out_dev, 0, sizeof(float), S(stream)), "cudaMemsetAsync");
    hf::k_divergence_max<<<592, 256, 0, S(stream)>>>(static_cast<const hf_scene*>(p->scenes_dev), s,
                                                    reinterpret_cast<unsigned*>(out_dev));
    HF_CUDA(cudaGetLastError(), "launch (divergence max)");
    return HF_OK;
}

int hf_speed_max(const hf_plan* p, int s, float* out_dev, void* stream) {
    int rc = check_plan(p);
    if (rc) return rc;
    if (s < 0 || s >= p->num_scenes || !out_dev) return fail(HF_ERR_ARG, "bad scene index or output");
    HF_CUDA(cudaMemsetAsync(out_dev, 0, sizeof(float), S(stream)), "cudaMemsetAsync");
    hf::k_speed_max<<<592, 256, 0, S(stream)>>>(static_cast<const hf_scene*>(p->scenes_dev), s,
                                               reinterpret_cast<unsigned*>(out_dev));
    HF_CUDA(cudaGetLastError(), "launch (speed max)");
    return HF_OK;
}

int hf_set_wait_limit(unsigned long long limit_ns, int absent_block) {
    if (limit_ns == 0 || limit_ns > 60000000000ull || absent_block < -1)
        return fail(HF_ERR_ARG, "hf_set_wait_limit: limit must be 1 ns .. 60 s, absent_block >= -1");
    int rc = hf::set_wait_limit(limit_ns, absent_block);
    if (rc) return fail(rc, "hf_set_wait_limit: cudaMemcpyToSymbol failed");
    return HF_OK;
}

int hf_k_divide_by(int count, const float* x, float y, float* out, void* stream) {
    if (count < 0 || (count > 0 && (!x || !out)) || !(y != 0.0f)) return fail(HF_ERR_ARG, "hf_k_divide_by: bad arguments");
    if (count == 0) return HF_OK;
    hf::k_divide_by<<<592, 256, 0, S(stream)>>>(count, x, y, out);
    HF_CUDA(cudaGetLastError(), "launch (divide_by)");
    return HF_OK;
}

int hf_k_laplacian(int n, double h, double alpha, double beta, const float* p, const float* ax, const float* ay,
                   const float* az, const float* y, float* out, void* stream) {
    if (n < 1 || !p || !ax || !ay || !az || !y || !out) return fail(HF_ERR_ARG, "hf_k_laplacian: bad arguments");
    hf::k_laplacian_plain<<<592, 256, 0, S(stream)>>>(n, (float)h, (float)alpha, (float)beta, p, ax, ay, az, y, out);
    HF_CUDA(cudaGetLastError(), "launch (laplacian)");
    return HF_OK;
}

int hf_k_heat_matvec(int n, double h, double dt, double alpha, double beta, const float* x, const float* kap,
                     const uint8_t* cell_flags, const float* y, float* out, void* stream) {
    if (n < 1 || !x || !kap || !cell_flags || !y || !out) return fail(HF_ERR_ARG, "hf_k_heat_matvec: bad arguments");
    hf::k_heat_matvec_plain<<<592, 256, 0, S(stream)>>>(n, (float)h, (float)dt, (float)alpha, (float)beta, x, kap, cell_flags,
                                                       y, out);
    HF_CUDA(cudaGetLastError(), "launch (heat matvec)");
    return HF_OK;
}

}  // extern "C"
