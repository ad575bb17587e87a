// hf_api.cu -- host side of the C ABI declared in include/heatflow_b200.h.
//
// Stateless apart from a per-device cache of SM count and cooperative-launch occupancy.  No function allocates device
// memory; the workspace layout below carves the caller's buffer.
#include <algorithm>
#include <cstdio>
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
    int occ_heat = 0, occ_pressure = 0;
    int occ_res[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};   // [heat][maxc]: blocks/SM at the variant's block size
    bool ready = false;
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
        HF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.occ_heat, hf::pcg_kernel(true), hf::kThreads, 0), "occupancy");
        HF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.occ_pressure, hf::pcg_kernel(false), hf::kThreads, 0),
                "occupancy");
        for (int h = 0; h < 2; ++h)
            for (int m = 1; m <= 3; ++m)
                HF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.occ_res[h][m], hf::pcg_resident_kernel(h == 1, m),
                                                                      256 * kResGroupsMax[m], 0),
                        "occupancy (resident)");
        if (!d.coop) return fail(HF_ERR_DEVICE, "device does not support cooperative launches");
        d.ready = true;
    }
    *out = &d;
    return HF_OK;
}

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

struct Layout {
    size_t head, chunk_begin, ctl, scene_count, partials, diag, total;
};

Layout layout(int S, int C) {
    Layout L{};
    size_t o = 0;
    L.head = o;                      // bar[2], live_count[2], err, pad -> 64 bytes
    o = align_up(o + 64, 256);
    L.chunk_begin = o;
    o = align_up(o + sizeof(int) * (size_t)(S + 1), 256);
    L.ctl = o;
    o = align_up(o + sizeof(hf::CgCtl) * (size_t)S, 256);
    L.scene_count = o;
    o = align_up(o + sizeof(unsigned) * (size_t)S, 256);
    L.partials = o;
    o = align_up(o + sizeof(double) * 6 * (size_t)C, 256);   // two partial buffers (phases A and B)
    L.diag = o;
    o = align_up(o + 64, 256);
    L.total = o;
    return L;
}

hf::Workspace workspace(const hf_plan* p) {
    const Layout L = layout(p->num_scenes, p->num_chunks);
    char* b = static_cast<char*>(p->workspace);
    hf::Workspace w;
    w.bar = reinterpret_cast<unsigned*>(b + L.head);
    w.live_count = w.bar + 2;
    w.err = reinterpret_cast<int*>(w.bar + 4);
    w.chunk_begin = reinterpret_cast<int*>(b + L.chunk_begin);
    w.ctl = reinterpret_cast<hf::CgCtl*>(b + L.ctl);
    w.scene_count = reinterpret_cast<unsigned*>(b + L.scene_count);
    w.partials = reinterpret_cast<double*>(b + L.partials);
    w.diag_bits = reinterpret_cast<unsigned*>(b + L.diag);
    return w;
}

int check_plan(const hf_plan* p) {
    if (!p || !p->scenes_host || !p->scenes_dev || !p->work_dev || !p->workspace) return fail(HF_ERR_ARG, "incomplete hf_plan");
    if (p->num_scenes <= 0 || p->num_scenes > hf::kMaxScenes) return fail(HF_ERR_ARG, "num_scenes out of range (1..1024)");
    if (p->workspace_bytes < layout(p->num_scenes, p->num_chunks).total)
        return fail(HF_ERR_WORKSPACE, "workspace smaller than hf_workspace_bytes()");
    return HF_OK;
}

inline cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }

bool any_flag(const hf_plan* p, unsigned f) {
    for (int s = 0; s < p->num_scenes; ++s)
        if ((p->scenes_host[s].flags & HF_FLAG_ACTIVE) && (p->scenes_host[s].flags & f)) return true;
    return false;
}

int launch_pcg(const hf_plan* p, bool heat, double dt, void* stream) {
    DeviceInfo* d = nullptr;
    int rc = device_info(&d);
    if (rc) return rc;
    if (p->num_chunks == 0) return HF_OK;
    hf::Workspace ws = workspace(p);
    const hf_scene* scenes = static_cast<const hf_scene*>(p->scenes_dev);
    const hf::WorkItem* work = static_cast<const hf::WorkItem*>(p->work_dev);
    int nc = p->num_chunks, ns = p->num_scenes;
    void* args[] = {(void*)&scenes, (void*)&work, (void*)&nc, (void*)&ns, (void*)&dt, (void*)&ws};
    // register-resident variant: one active scene whose chunks fit one block per SM
    int active = 0;
    for (int s = 0; s < p->num_scenes; ++s) active += (p->scenes_host[s].flags & HF_FLAG_ACTIVE) ? 1 : 0;
    if (active == 1 && !(p->options & HF_PLAN_STREAMING_CG)) {
        const int G = p->num_chunks < d->sms ? p->num_chunks : d->sms;
        const int cpb = (p->num_chunks + G - 1) / G;
        for (int m = 1; m <= 3; ++m) {
            const int groups = (cpb + m - 1) / m;
            if (groups > kResGroupsMax[m] || d->occ_res[heat ? 1 : 0][m] < 1) continue;
            HF_CUDA(cudaMemsetAsync(ws.bar, 0, 64, S(stream)), "cudaMemsetAsync(barrier)");
            HF_CUDA(cudaLaunchCooperativeKernel(hf::pcg_resident_kernel(heat, m), dim3(G), dim3(256 * groups), args, 0, S(stream)),
                    "cooperative launch (resident CG)");
            return HF_OK;
        }
    }
    const int occ = heat ? d->occ_heat : d->occ_pressure;
    if (occ <= 0) return fail(HF_ERR_DEVICE, "persistent CG kernel does not fit on an SM");
    int per_sm = occ < 2 ? occ : 2;
    int grid = p->persistent_blocks > 0 ? p->persistent_blocks : d->sms * per_sm;
    if (grid > d->sms * occ) grid = d->sms * occ;
    if (grid > p->num_chunks) grid = p->num_chunks;
    // every block keeps the scalars of the scenes its contiguous chunk range touches (at most 32)
    std::vector<int> begin(p->num_scenes + 1, 0);
    for (int s = 0; s < p->num_scenes; ++s) {
        const hf_scene& sc = p->scenes_host[s];
        begin[s + 1] = begin[s] + ((sc.flags & HF_FLAG_ACTIVE) ? hf_chunks_for(sc.n) : 0);
    }
    if (begin[p->num_scenes] != p->num_chunks) return fail(HF_ERR_ARG, "plan changed since hf_plan_upload");
    for (int b = 0; b < grid; ++b) {
        const int c0 = (int)(((long long)p->num_chunks * b) / grid), c1 = (int)(((long long)p->num_chunks * (b + 1)) / grid);
        if (c1 <= c0) continue;
        const int s0 = (int)(std::upper_bound(begin.begin(), begin.end(), c0) - begin.begin()) - 1;
        const int s1 = (int)(std::upper_bound(begin.begin(), begin.end(), c1 - 1) - begin.begin()) - 1;
        if (s1 - s0 + 1 > 32) return fail(HF_ERR_ARG, "more than 32 scenes in one block's chunk range: use more blocks");
    }
    // barrier counters, live counts and the timeout flag start at zero for every solve
    HF_CUDA(cudaMemsetAsync(ws.bar, 0, 64, S(stream)), "cudaMemsetAsync(barrier)");
    const void* fn = hf::pcg_kernel(heat);
    HF_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(hf::kThreads), args, 0, S(stream)), "cooperative launch (CG)");
    return HF_OK;
}

}  // namespace

extern "C" {

int hf_abi_version(void) { return HF_ABI_VERSION; }

const char* hf_last_error(void) { return g_err.c_str(); }

int hf_cells_per_chunk(void) { return hf::kChunk; }

int hf_chunks_for(int n) {
    if (n <= 0) return 0;
    const long long N = (long long)n * n * n;
    return (int)((N + hf::kChunk - 1) / hf::kChunk);
}

size_t hf_workspace_bytes(int num_scenes, int num_chunks) { return layout(num_scenes, num_chunks).total; }

int hf_plan_upload(hf_plan* p, void* stream) {
    if (!p || !p->scenes_host || !p->scenes_dev || !p->work_dev || !p->workspace) return fail(HF_ERR_ARG, "incomplete hf_plan");
    if (p->num_scenes <= 0 || p->num_scenes > hf::kMaxScenes) return fail(HF_ERR_ARG, "num_scenes out of range (1..1024)");
    std::vector<hf::WorkItem> work;
    std::vector<int> begin(p->num_scenes + 1, 0);
    for (int s = 0; s < p->num_scenes; ++s) {
        const hf_scene& sc = p->scenes_host[s];
        begin[s] = (int)work.size();
        if (!(sc.flags & HF_FLAG_ACTIVE)) continue;
        if (sc.n < 2 || sc.n > 1024) return fail(HF_ERR_ARG, "scene edge n out of range (2..1024)");
        if (!sc.state) return fail(HF_ERR_ARG, "scene without a state block");
        const long long N = (long long)sc.n * sc.n * sc.n;
        for (long long f = 0; f < N; f += hf::kChunk) work.push_back(hf::WorkItem{s, (int)f});
    }
    begin[p->num_scenes] = (int)work.size();
    p->num_chunks = (int)work.size();
    const Layout L = layout(p->num_scenes, p->num_chunks);
    if (p->workspace_bytes < L.total) return fail(HF_ERR_WORKSPACE, "workspace smaller than hf_workspace_bytes()");
    HF_CUDA(cudaMemsetAsync(p->workspace, 0, L.total, S(stream)), "cudaMemsetAsync(workspace)");
    HF_CUDA(cudaMemcpyAsync(p->scenes_dev, p->scenes_host, sizeof(hf_scene) * p->num_scenes, cudaMemcpyHostToDevice, S(stream)),
            "upload scene table");
    if (!work.empty())
        HF_CUDA(cudaMemcpyAsync(p->work_dev, work.data(), sizeof(hf::WorkItem) * work.size(), cudaMemcpyHostToDevice, S(stream)),
                "upload work table");
    char* b = static_cast<char*>(p->workspace);
    HF_CUDA(cudaMemcpyAsync(b + L.chunk_begin, begin.data(), sizeof(int) * begin.size(), cudaMemcpyHostToDevice, S(stream)),
            "upload chunk table");
    HF_CUDA(cudaStreamSynchronize(S(stream)), "cudaStreamSynchronize(plan upload)");
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
        hf::k_footprint<<<(sc.n_particles + hf::kThreads - 1) / hf::kThreads, hf::kThreads, 0, S(stream)>>>(scenes, s);
        hf::k_scatter<<<(sc.n_particles + hf::kThreads - 1) / hf::kThreads, hf::kThreads, 0, S(stream)>>>(scenes, s);
    }
    if (p->num_chunks) {
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
    hf::k_prestage<<<p->num_chunks, hf::kThreads, 0, S(stream)>>>(scenes, work, dt);
    hf::k_advect_T<<<p->num_chunks, hf::kThreads, 0, S(stream)>>>(scenes, work, dt);
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
    if (!p->num_chunks) return HF_OK;
    hf::k_face_stage<<<p->num_chunks, hf::kThreads, 0, S(stream)>>>(static_cast<const hf_scene*>(p->scenes_dev),
                                                                   static_cast<const hf::WorkItem*>(p->work_dev), dt);
    HF_CUDA(cudaGetLastError(), "launch (face stage)");
    return HF_OK;
}

int hf_divergence_stage(const hf_plan* p, double dt, void* stream) {
    int rc = check_plan(p);
    if (rc) return rc;
    if (!p->num_chunks) return HF_OK;
    hf::k_divergence<<<p->num_chunks, hf::kThreads, 0, S(stream)>>>(static_cast<const hf_scene*>(p->scenes_dev),
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
