// hf_noalloc.cu -- hf_pressure_solve_noalloc: the pressure stage of one scene without any device allocation.
//
// Some callers cannot call cudaMalloc: code that runs where an allocator is not available or not allowed -- inside an
// allocator callback, under a memory pool or budget that the caller does not own, or in a host that pre-plans all its
// device memory up front and forbids allocations once it runs.  This entry point serves them: the caller passes the
// scene's inputs and outputs, and everything else the solve needs (scene record, work tables, CG workspace and CG
// vectors) lives in one file-scope device array of fixed size, `g_noalloc_scratch`, which every GPU that loads the
// library holds until the process exits.
//
// The array is shared by every call on a device and keeps the last call's contents; each call clears what must
// start at zero.  Calls whose work overlaps on the GPU (different streams, or streams without ordering between them)
// race on the array.
#include <cstring>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <mutex>

#include "hf_device.cuh"
#include "hf_kernels.cuh"

namespace {

constexpr int kMaxEdge = 64;                           // scenes up to 64^3 cells
constexpr size_t kScratchBytes = 9u * 1024u * 1024u;   // 9 MiB, enough for kMaxEdge (checked in layout())

__device__ __align__(256) static unsigned char g_noalloc_scratch[kScratchBytes];

size_t up256(size_t x) { return (x + 255) / 256 * 256; }

struct ScratchLayout {
    size_t rec, state, chunks, tiles, ws, ws_bytes, qzero, vec[7], total;
};

ScratchLayout layout(int n, int C, int T) {
    ScratchLayout L{};
    const size_t N = (size_t)n * n * n, NF = (size_t)(n + 1) * n * n;
    size_t o = 0;
    L.rec = o;
    o = up256(o + sizeof(hf_scene));
    L.state = o;
    o = up256(o + sizeof(hf_scene_state));
    L.chunks = o;
    o = up256(o + sizeof(hf::WorkItem) * (size_t)C);
    L.tiles = o;
    o = up256(o + sizeof(hf::TileItem) * (size_t)T);
    L.ws = o;
    L.ws_bytes = hf_workspace_bytes(1, C, T);
    o = up256(o + L.ws_bytes);
    L.qzero = o;
    o = up256(o + sizeof(float) * NF);
    for (int i = 0; i < 7; ++i) {   // rhs, pdiag, cg_r, cg_z, cg_p[0], cg_p[1], cg_Ap
        L.vec[i] = o;
        o = up256(o + sizeof(float) * N);
    }
    L.total = o;
    return L;
}

std::mutex g_mu;
// Address of the scratch array per device, with the context it was looked up in: a cached address belongs to one
// context and does not survive cudaDeviceReset (or another driver-API context on the device), so the lookup is
// repeated whenever the current context differs from the cached one.
struct BaseCache {
    CUcontext ctx = nullptr;
    unsigned char* base = nullptr;
};
BaseCache g_base[64];
PFN_cuCtxGetCurrent_v4000 g_ctx_current = nullptr;

// Device address of the scratch array on the current device (looked up once per device and context).
int scratch_base(unsigned char** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return HF_ERR_CUDA;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ctx_current) {
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", reinterpret_cast<void**>(&g_ctx_current), cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !g_ctx_current)
            return HF_ERR_CUDA;
    }
    // no context is current yet when the runtime has not touched this device; the lookup below creates it
    CUcontext ctx = nullptr;
    if (g_ctx_current(&ctx) != CUDA_SUCCESS) return HF_ERR_CUDA;
    BaseCache& c = g_base[dev];
    if (!c.base || !ctx || c.ctx != ctx) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return HF_ERR_CUDA;
        if (g_ctx_current(&ctx) != CUDA_SUCCESS || !ctx) return HF_ERR_CUDA;
        c.base = static_cast<unsigned char*>(p);
        c.ctx = ctx;
    }
    *out = c.base;
    return HF_OK;
}

// Writes the scene record, the chunk and tile tables and the zeroed state, workspace header and zero flux into the
// scratch array (one launch, no host memory involved).
__global__ void k_noalloc_setup(hf_scene rec, unsigned char* base, ScratchLayout L, int C, int T, int zero_q) {
    const int n = rec.n;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    if (tid == 0) {
        *reinterpret_cast<hf_scene*>(base + L.rec) = rec;
        hf_scene_state* st = reinterpret_cast<hf_scene_state*>(base + L.state);
        memset(st, 0, sizeof(hf_scene_state));
    }
    // workspace: everything before the partial buffers starts at zero; then the one-scene offset tables
    for (size_t b = tid; b < L.ws_bytes; b += stride) base[L.ws + b] = 0;
    hf::WorkItem* chunks = reinterpret_cast<hf::WorkItem*>(base + L.chunks);
    for (int c = tid; c < C; c += stride) chunks[c] = hf::WorkItem{0, c * hf::kChunk};
    const int ti = (n + hf::kTI - 1) / hf::kTI, tk = (n + hf::kTK - 1) / hf::kTK;
    hf::TileItem* tiles = reinterpret_cast<hf::TileItem*>(base + L.tiles);
    for (int c = tid; c < T; c += stride)   // same order as hf_plan_upload: k fastest, then i, then j
        tiles[c] = hf::TileItem{0, ((c / tk) % ti) * hf::kTI, (c / (tk * ti)) * hf::kTJ, (c % tk) * hf::kTK};
    if (zero_q) {
        float* q = reinterpret_cast<float*>(base + L.qzero);
        const size_t NF = (size_t)(n + 1) * n * n;
        for (size_t f = tid; f < NF; f += stride) q[f] = 0.0f;
    }
}

__global__ void k_noalloc_offsets(int* cb, int* tb, int C, int T) {
    cb[0] = 0;
    cb[1] = C;
    tb[0] = 0;
    tb[1] = T;
}

}  // namespace

extern "C" size_t hf_noalloc_scratch_bytes(void) { return kScratchBytes; }

extern "C" int hf_noalloc_max_edge(void) { return kMaxEdge; }

extern "C" int hf_pressure_solve_noalloc(int n, double h, double rho, double dt, double cg_tol, int cg_max_iter,
                                         float* u, float* v, float* w, const float* ax, const float* ay, const float* az,
                                         const float* qx, const float* qy, const float* qz, float* p,
                                         hf_scene_state* state_out, void* stream) {
    if (n < 2 || n > kMaxEdge)
        return hf::set_error(HF_ERR_ARG, "hf_pressure_solve_noalloc: scene edge n must be 2..64 (its fixed 9 MiB scratch "
                                         "array holds no larger scene); use hf_pressure_solve with caller-owned buffers");
    if (!u || !v || !w || !ax || !ay || !az || !p)
        return hf::set_error(HF_ERR_ARG, "hf_pressure_solve_noalloc: null field pointer");
    if ((qx == nullptr) != (qy == nullptr) || (qx == nullptr) != (qz == nullptr))
        return hf::set_error(HF_ERR_ARG, "hf_pressure_solve_noalloc: pass all of qx, qy, qz or none");
    const int C = hf_chunks_for(n), T = hf_tiles_for(n);
    const ScratchLayout L = layout(n, C, T);
    if (L.total > kScratchBytes) return hf::set_error(HF_ERR_ARG, "hf_pressure_solve_noalloc: scratch array too small");
    unsigned char* base = nullptr;
    int rc = scratch_base(&base);
    if (rc) return hf::set_error(rc, "hf_pressure_solve_noalloc: cudaGetSymbolAddress of the scratch array failed");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float* vec[7];
    for (int i = 0; i < 7; ++i) vec[i] = reinterpret_cast<float*>(base + L.vec[i]);
    float* qz0 = reinterpret_cast<float*>(base + L.qzero);

    hf_scene rec;
    std::memset(&rec, 0, sizeof rec);
    rec.n = n;
    rec.flags = HF_FLAG_ACTIVE;
    rec.cg_max_iter = cg_max_iter;
    rec.h = h;
    rec.rho = rho;
    rec.cg_tol = cg_tol;
    rec.u[0] = rec.u[1] = u;   // both parities name the caller's arrays: read and projected in place
    rec.v[0] = rec.v[1] = v;
    rec.w[0] = rec.w[1] = w;
    rec.ax = const_cast<float*>(ax);
    rec.ay = const_cast<float*>(ay);
    rec.az = const_cast<float*>(az);
    rec.qx = const_cast<float*>(qx ? qx : qz0);
    rec.qy = const_cast<float*>(qy ? qy : qz0);
    rec.qz = const_cast<float*>(qz ? qz : qz0);
    rec.p = p;
    rec.rhs = vec[0];
    rec.pdiag = vec[1];
    rec.cg_r = vec[2];
    rec.cg_z = vec[3];
    rec.cg_p[0] = vec[4];
    rec.cg_p[1] = vec[5];
    rec.cg_Ap = vec[6];
    rec.state = reinterpret_cast<hf_scene_state*>(base + L.state);

    k_noalloc_setup<<<64, 256, 0, s>>>(rec, base, L, C, T, qx == nullptr);
    if (cudaGetLastError() != cudaSuccess) return hf::set_error(HF_ERR_CUDA, "hf_pressure_solve_noalloc: set-up launch failed");
    // the workspace's offset tables (after the zeroing above): layout of hf_workspace_bytes(1, C, T)
    hf_plan plan;
    std::memset(&plan, 0, sizeof plan);
    plan.num_scenes = 1;
    plan.num_chunks = C;
    plan.num_tiles = T;
    plan.scenes_host = &rec;
    plan.scenes_dev = base + L.rec;
    plan.work_dev = base + L.chunks;
    plan.tiles_dev = base + L.tiles;
    plan.workspace = base + L.ws;
    plan.workspace_bytes = L.ws_bytes;
    plan.options = HF_PLAN_STREAMING_CG;
    int *cbeg = nullptr, *tbeg = nullptr;
    hf::plan_offset_tables(&plan, &cbeg, &tbeg);
    k_noalloc_offsets<<<1, 1, 0, s>>>(cbeg, tbeg, C, T);
    if (cudaGetLastError() != cudaSuccess) return hf::set_error(HF_ERR_CUDA, "hf_pressure_solve_noalloc: set-up launch failed");
    if ((rc = hf_divergence_stage(&plan, dt, stream))) return rc;
    if ((rc = hf_pressure_cg(&plan, dt, stream))) return rc;
    if (state_out && cudaMemcpyAsync(state_out, rec.state, sizeof(hf_scene_state), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        return hf::set_error(HF_ERR_CUDA, "hf_pressure_solve_noalloc: copy of the solve statistics failed");
    return HF_OK;
}
