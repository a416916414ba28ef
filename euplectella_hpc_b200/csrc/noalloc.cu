// Momentum-exchange force for callers that cannot allocate device memory.
//
// eup_get_forces reduces through per-block partial sums that live in buffers
// the handle allocated.  Some callers can hold no handle and must not let a
// library allocate: a Fortran driver whose a01..a19 and obs already sit on the
// GPU under its own OpenACC data region (the reference's GPU build) and whose
// runtime owns the device memory, or a code that hands out a fixed device-memory
// budget through its own allocator, where an extra cudaMalloc would fail or
// stall every stream on the device.  This
// entry point reads the caller's device arrays in the reference's haloed
// layout and writes the force to the caller's device memory; its only scratch
// is the file-scope array below, of fixed size.  The CUDA runtime loads the
// library's device code lazily (CUDA_MODULE_LOADING=LAZY is the default), so
// the array is created on a device by the first call there: a caller with a
// fixed device-memory budget makes one call (any small lattice) before its own
// allocator takes that budget.
#include <cuda_runtime.h>

#include <string>

#include "../../include/eup.h"
#include "lbm_common.cuh"

void eup_internal_set_error(const std::string& msg);

namespace {

// One FP64 partial force per z-plane plus the completion counter.  Every GPU
// on which the entry point has been called holds this array (about 96 KiB)
// until the process exits.  All calls share it, so calls that overlap on the GPU (different
// streams, or different host threads on one device) race on it.
constexpr int kNoAllocMaxPlanes = 4096;
struct NoAllocScratch {
    double plane[kNoAllocMaxPlanes][3];
    unsigned int done;
};
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// The caller's 19 population arrays, passed by value to the kernel.
template <typename T>
struct Pops19 {
    const T* p[19];
};

// Device address of the scratch on the current device.  In host code the
// symbol is only a host-side stand-in; the address is looked up on every call
// (cheap next to the launch), so it stays right after a device reset or a
// runtime shutdown and re-initialisation reloads the module elsewhere.
cudaError_t scratch_for_current_device(NoAllocScratch** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    *out = static_cast<NoAllocScratch*>(p);
    return cudaSuccess;
}

// One block per z-plane k: F = sum over fluid nodes y of the plane and
// directions q with solid neighbour wrap(y + c_q) of 2 c_q a_q(y) (the same
// definition as eup_get_forces).  Plane partials are added in k order by the
// last block, so the result does not depend on scheduling.
template <typename T>
__global__ void __launch_bounds__(256) k_mem_force_noalloc(int l, int m, int n, int per_x, int per_y, int per_z,
                                                           Pops19<T> pops, const int32_t* obs,
                                                           NoAllocScratch* scr, double* force) {
    const int k = blockIdx.x + 1;
    const int64_t L2 = l + 2, M2 = m + 2;
    double f[3] = {0.0, 0.0, 0.0};
    for (int64_t t = threadIdx.x; t < (int64_t)l * m; t += blockDim.x) {
        const int i = (int)(t % l) + 1, j = (int)(t / l) + 1;
        const int64_t o = (int64_t)(i - 1) + (int64_t)l * ((j - 1) + (int64_t)m * (k - 1));
        if (obs[o] == 1) continue;
#pragma unroll
        for (int q = 0; q < 18; ++q) {
            int ni = i + eup::cx_of(q), nj = j + eup::cy_of(q), nk = k + eup::cz_of(q);
            if (per_x) ni = ni < 1 ? ni + l : (ni > l ? ni - l : ni);
            if (per_y) nj = nj < 1 ? nj + m : (nj > m ? nj - m : nj);
            if (per_z) nk = nk < 1 ? nk + n : (nk > n ? nk - n : nk);
            if (ni < 1 || ni > l || nj < 1 || nj > m || nk < 1 || nk > n) continue;
            if (obs[(int64_t)(ni - 1) + (int64_t)l * ((nj - 1) + (int64_t)m * (nk - 1))] != 1) continue;
            const double v = (double)pops.p[q][(int64_t)i + L2 * ((int64_t)j + M2 * k)];
            f[0] += 2.0 * eup::cx_of(q) * v;
            f[1] += 2.0 * eup::cy_of(q) * v;
            f[2] += 2.0 * eup::cz_of(q) * v;
        }
    }
    __shared__ double sh[8][3];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 3; ++c)
        for (int s = 16; s > 0; s >>= 1) f[c] += __shfl_down_sync(0xffffffffu, f[c], s);
    if (lane == 0)
        for (int c = 0; c < 3; ++c) sh[warp][c] = f[c];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int c = 0; c < 3; ++c) {
            double s = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[w][c];
            scr->plane[blockIdx.x][c] = s;
        }
        __threadfence();
        last = (atomicAdd(&scr->done, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    for (int c = 0; c < 3; ++c) {
        double s = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) s += ((volatile double*)scr->plane[b])[c];
        force[c] = s;
    }
    scr->done = 0u;
}

}  // namespace

extern "C" int eup_mem_force_noalloc(int32_t l, int32_t m, int32_t n, const int32_t bc[6],
                                     const void* const pops[19], int32_t elem_bytes, const int32_t* obs,
                                     double* force, void* stream) {
    if (l < 1 || m < 1 || n < 1 || !bc || !pops || !obs || !force || (elem_bytes != 4 && elem_bytes != 8)) {
        eup_internal_set_error("eup_mem_force_noalloc: bad argument");
        return EUP_ERR_INVALID_ARG;
    }
    if (n > kNoAllocMaxPlanes) {
        eup_internal_set_error("eup_mem_force_noalloc: lz = " + std::to_string(n) + " exceeds the maximum of " +
                               std::to_string(kNoAllocMaxPlanes) + " z-planes held by its fixed scratch");
        return EUP_ERR_UNSUPPORTED;
    }
    if ((int64_t)l * m > 2147483647LL) {
        eup_internal_set_error("eup_mem_force_noalloc: more than 2^31-1 nodes per z-plane");
        return EUP_ERR_UNSUPPORTED;
    }
    for (int q = 0; q < 19; ++q)
        if (!pops[q]) {
            eup_internal_set_error("eup_mem_force_noalloc: null population array");
            return EUP_ERR_INVALID_ARG;
        }
    NoAllocScratch* scr = nullptr;
    cudaError_t e = scratch_for_current_device(&scr);
    if (e != cudaSuccess) {
        eup_internal_set_error(std::string("eup_mem_force_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        return EUP_ERR_CUDA;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the counter must start at zero; the plane partials are all overwritten
    e = cudaMemsetAsync(&scr->done, 0, sizeof(unsigned int), st);
    const int per_x = (bc[EUP_FRONT] == 0 && bc[EUP_REAR] == 0);
    const int per_y = (bc[EUP_RIGHT] == 0 && bc[EUP_LEFT] == 0);
    const int per_z = (bc[EUP_UP] == 0 && bc[EUP_DOWN] == 0);
    if (e == cudaSuccess) {
        if (elem_bytes == 4) {
            Pops19<float> p;
            for (int q = 0; q < 19; ++q) p.p[q] = static_cast<const float*>(pops[q]);
            k_mem_force_noalloc<float><<<n, 256, 0, st>>>(l, m, n, per_x, per_y, per_z, p, obs, scr, force);
        } else {
            Pops19<double> p;
            for (int q = 0; q < 19; ++q) p.p[q] = static_cast<const double*>(pops[q]);
            k_mem_force_noalloc<double><<<n, 256, 0, st>>>(l, m, n, per_x, per_y, per_z, p, obs, scr, force);
        }
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        eup_internal_set_error(std::string("eup_mem_force_noalloc: ") + cudaGetErrorString(e));
        return EUP_ERR_CUDA;
    }
    return EUP_OK;
}
