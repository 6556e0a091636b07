// Ghost-plane exchange of a z-slab decomposition: packs chosen population slots of whole z-planes of
// a PDF field into contiguous buffers and unpacks them back, one launch for every plane of an
// exchange (lbmpy's communication slices, advanced_streaming/communication.py:122-183, restricted
// to the z faces).  The element type only matters through its size: plain copies of 2, 4 or 8 bytes.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/lbm_b200.h"

namespace lbm {
int abi_fail(int code, const char* fmt, ...);
}

namespace {

struct HaloJobs {
    LbmHaloJob job[LBM_HALO_MAX_JOBS];
    int n_jobs;
};

template <class T>
__global__ void __launch_bounds__(256) k_halo_copy(T* pdfs, long long sy, long long sz, long long sq, int nx, int ny,
                                                  const HaloJobs jobs) {
    const LbmHaloJob& j = jobs.job[blockIdx.y];
    const long long plane = (long long)nx * ny;
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= plane * j.n_slots) return;
    const int k = int(e / plane);
    const long long c = e - k * plane;
    const int x = int(c % nx), y = int(c / nx);
    T* f = pdfs + x + y * sy + (long long)j.z * sz + (long long)j.slots[k] * sq;
    T* b = static_cast<T*>(j.buffer) + e;
    if (j.unpack) *f = *b;
    else *b = *f;
}

}  // namespace

extern "C" int lbm_halo_copy(void* pdfs, const int64_t strides[4], int32_t q, int32_t nx_ext, int32_t ny_ext,
                             int32_t nz_ext, int32_t elem_size, const LbmHaloJob* jobs, int32_t n_jobs, void* stream) {
    using lbm::abi_fail;
    if (pdfs == nullptr || strides == nullptr || jobs == nullptr)
        return abi_fail(LBM_E_INVALID, "pdfs, strides and jobs must not be NULL");
    if (n_jobs < 1 || n_jobs > LBM_HALO_MAX_JOBS)
        return abi_fail(LBM_E_INVALID, "n_jobs must be in [1, %d]", LBM_HALO_MAX_JOBS);
    if (elem_size != 2 && elem_size != 4 && elem_size != 8)
        return abi_fail(LBM_E_INVALID, "elem_size must be 2, 4 or 8 bytes");
    if (nx_ext < 1 || ny_ext < 1 || nz_ext < 1) return abi_fail(LBM_E_INVALID, "plane extents must be positive");
    if (q < 1 || q > 27) return abi_fail(LBM_E_INVALID, "q must be in [1, 27]");
    if (strides[0] != 1 || strides[1] < nx_ext || strides[2] < strides[1] * ny_ext ||
        strides[3] < strides[2] * nz_ext)
        return abi_fail(LBM_E_INVALID, "strides must be {1, sy >= nx, sz >= sy * ny, sq >= sz * nz} elements");
    HaloJobs h;
    memset(&h, 0, sizeof(h));
    h.n_jobs = n_jobs;
    int max_slots = 0;
    for (int k = 0; k < n_jobs; ++k) {
        const LbmHaloJob& j = jobs[k];
        if (j.buffer == nullptr) return abi_fail(LBM_E_INVALID, "job %d has no buffer", k);
        if (j.z < 0 || j.z >= nz_ext) return abi_fail(LBM_E_INVALID, "job %d: plane %d outside [0, %d)", k, j.z, nz_ext);
        if (j.n_slots < 1 || j.n_slots > q) return abi_fail(LBM_E_INVALID, "job %d: n_slots must be in [1, q]", k);
        for (int s = 0; s < j.n_slots; ++s)
            if (j.slots[s] < 0 || j.slots[s] >= q)
                return abi_fail(LBM_E_INVALID, "job %d: slot %d out of range", k, j.slots[s]);
        h.job[k] = j;
        if (j.n_slots > max_slots) max_slots = j.n_slots;
    }
    const long long work = (long long)nx_ext * ny_ext * max_slots;
    const dim3 grid((unsigned)((work + 255) / 256), (unsigned)n_jobs);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (elem_size) {
        case 2: k_halo_copy<uint16_t><<<grid, 256, 0, s>>>(static_cast<uint16_t*>(pdfs), strides[1], strides[2],
                                                          strides[3], nx_ext, ny_ext, h); break;
        case 4: k_halo_copy<uint32_t><<<grid, 256, 0, s>>>(static_cast<uint32_t*>(pdfs), strides[1], strides[2],
                                                          strides[3], nx_ext, ny_ext, h); break;
        default: k_halo_copy<uint64_t><<<grid, 256, 0, s>>>(static_cast<uint64_t*>(pdfs), strides[1], strides[2],
                                                           strides[3], nx_ext, ny_ext, h); break;
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LBM_OK : abi_fail(LBM_E_CUDA, "halo copy launch: %s", cudaGetErrorString(e));
}
