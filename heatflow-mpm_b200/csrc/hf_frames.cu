// hf_frames.cu -- one output frame packed on the device.
//
// A frame of the reference's scene driver (scripts/run_scene.py:31-40, fields of solver.py:105-110 frame_dict) holds
// grid_T as binary16 [n^3], the cell-centred air velocity (grid.py:156-162) as binary16 [n^3, 3] and the particles'
// temperature and melt fraction as binary16.  k_pack_frame converts them in one launch into caller buffers (one
// contiguous block if the caller lays them out so), so that a single asynchronous copy moves a frame to the host while
// the next substeps run.  Conversions round to nearest even, as numpy's astype(float16) does.
#include <cuda_fp16.h>

#include "hf_device.cuh"
#include "hf_kernels.cuh"

namespace hf {

__global__ void __launch_bounds__(kThreads) k_pack_frame(const hf_scene* __restrict__ scenes, int s, __half* grid_T,
                                                         __half* air_u, __half* temp, __half* melt) {
    const hf_scene& S = scenes[s];
    const int n = S.n, N = n * n * n, par = S.state->parity, P = S.n_particles;
    const float* T = S.T[par];
    const float *u = S.u[par], *v = S.v[par], *w = S.w[par];
    const int stride = gridDim.x * blockDim.x;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < N; t += stride) {
        if (grid_T) grid_T[t] = __float2half_rn(T[t]);
        if (air_u) {
            const int k = t % n, q = t / n, j = q % n, i = q / n;
            const int fu = (i * n + j) * n + k, fv = (i * (n + 1) + j) * n + k, fw = (i * n + j) * (n + 1) + k;
            air_u[3 * t + 0] = __float2half_rn(__fmul_rn(0.5f, __fadd_rn(u[fu], u[fu + n * n])));
            air_u[3 * t + 1] = __float2half_rn(__fmul_rn(0.5f, __fadd_rn(v[fv], v[fv + n])));
            air_u[3 * t + 2] = __float2half_rn(__fmul_rn(0.5f, __fadd_rn(w[fw], w[fw + 1])));
        }
    }
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += stride) {
        if (temp) temp[p] = __float2half_rn(S.ptemp[p]);
        if (melt) melt[p] = __float2half_rn(S.pmelt[p]);
    }
}

// The current buffer (device-side parity) of T, u, v or w of scene s, copied into `out`.
__global__ void __launch_bounds__(kThreads) k_current_field(const hf_scene* __restrict__ scenes, int s, int which,
                                                            float* __restrict__ out) {
    const hf_scene& S = scenes[s];
    const int n = S.n, par = S.state->parity;
    const long long N = (long long)n * n * n, F = (long long)(n + 1) * n * n;
    const float* src = which == 0 ? S.T[par] : which == 1 ? S.u[par] : which == 2 ? S.v[par] : S.w[par];
    const long long count = which == 0 ? N : F;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < count; t += (long long)gridDim.x * blockDim.x)
        out[t] = src[t];
}

}  // namespace hf

extern "C" int hf_current_field(const hf_plan* p, int s, int which, float* out, void* stream) {
    if (!p || !p->scenes_dev || !p->scenes_host || s < 0 || s >= p->num_scenes || which < 0 || which > 3 || !out)
        return hf::set_error(HF_ERR_ARG, "hf_current_field: bad plan, scene index, field or output");
    hf::k_current_field<<<592, hf::kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const hf_scene*>(p->scenes_dev), s, which, out);
    if (cudaGetLastError() != cudaSuccess) return hf::set_error(HF_ERR_CUDA, "hf_current_field: launch failed");
    return HF_OK;
}

extern "C" int hf_pack_frame(const hf_plan* p, int s, void* grid_T, void* air_u, void* temp, void* melt, void* stream) {
    if (!p || !p->scenes_dev || !p->scenes_host || s < 0 || s >= p->num_scenes)
        return hf::set_error(HF_ERR_ARG, "hf_pack_frame: bad plan or scene index");
    const hf_scene& sc = p->scenes_host[s];
    if ((temp || melt) && sc.n_particles > 0 && (!sc.ptemp || !sc.pmelt))
        return hf::set_error(HF_ERR_ARG, "hf_pack_frame: particle outputs requested for a scene without particles");
    hf::k_pack_frame<<<592, hf::kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const hf_scene*>(p->scenes_dev), s, static_cast<__half*>(grid_T), static_cast<__half*>(air_u),
        static_cast<__half*>(temp), static_cast<__half*>(melt));
    if (cudaGetLastError() != cudaSuccess) return hf::set_error(HF_ERR_CUDA, "hf_pack_frame: launch failed");
    return HF_OK;
}
