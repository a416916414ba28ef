// Set-up kernels for the solid mask (CODE/SRC/build.obs.F90 feeds
// CODE/SRC/bcond.obs.F90): bit packing, the device voxeliser, link
// classification, the ordered list of solid voxels that touch fluid or halo,
// and the obstacle-file records.
#include <algorithm>

#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "geometry.h"
#include "internal.h"

namespace eup {

namespace {

// One thread per 32-bit word of a row: bit b of word w of row (j,k) is obs(32w+b+1, j, k) == 1.
__global__ void k_build_mask(const int32_t* obs, Geo g, uint32_t* bits, int wpr) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t rows = (int64_t)g.m * g.n;
    if (t >= rows * wpr) return;
    const int64_t row = t / wpr;
    const int w = (int)(t % wpr);
    uint32_t word = 0;
    for (int b = 0; b < 32; ++b) {
        const int i0 = 32 * w + b;  // 0-based i
        if (i0 < g.l && obs[row * g.l + i0] == 1) word |= 1u << b;
    }
    bits[t] = word;
}

// Solid voxel with at least one of its 18 neighbours not an interior solid voxel.
__global__ void k_flag_boundary_solid(Geo g, Mask mk, uint8_t* flags) {
    const int64_t lin = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (lin >= g.N) return;
    const int i = (int)(lin % g.l) + 1, j = (int)((lin / g.l) % g.m) + 1, k = (int)(lin / g.lm) + 1;
    uint8_t f = 0;
    if (mk.solid(g, i, j, k)) {
#pragma unroll
        for (int q = 0; q < 18; ++q)
            if (!mk.solid(g, i + cx_of(q), j + cy_of(q), k + cz_of(q))) f = 1;
    }
    flags[lin] = f;
}

// bit q: fluid node whose upstream neighbour x - c_q is an interior solid voxel; bit 31: solid.
__global__ void k_links(Geo g, Mask mk, uint32_t* links) {
    const int64_t lin = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (lin >= g.N) return;
    const int i = (int)(lin % g.l) + 1, j = (int)((lin / g.l) % g.m) + 1, k = (int)(lin / g.lm) + 1;
    uint32_t w = 0;
    if (mk.solid(g, i, j, k)) {
        w = 0x80000000u;
    } else {
#pragma unroll
        for (int q = 0; q < 18; ++q)
            if (mk.solid(g, i - cx_of(q), j - cy_of(q), k - cz_of(q))) w |= 1u << q;
    }
    links[lin] = w;
}

__global__ void k_bsolid_links(Geo g, Mask mk, int per_x, int per_y, int per_z, const int32_t* list, int64_t n,
                               uint64_t* links) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int64_t lin = list[t];
    const int i = (int)(lin % g.l) + 1, j = (int)((lin / g.l) % g.m) + 1, k = (int)(lin / g.lm) + 1;
    uint64_t w = 0;
    for (int q = 0; q < 18; ++q) {
        const int ni = i + cx_of(q), nj = j + cy_of(q), nk = k + cz_of(q);
        if (g.interior(ni, nj, nk)) {
            if (!mk.solid(g, ni, nj, nk)) w |= 1ull << q;
        } else {
            w |= 1ull << (18 + q);
            int wi = ni, wj = nj, wk = nk;
            if (per_x) wi = wi < 1 ? wi + g.l : (wi > g.l ? wi - g.l : wi);
            if (per_y) wj = wj < 1 ? wj + g.m : (wj > g.m ? wj - g.m : wj);
            if (per_z) wk = wk < 1 ? wk + g.n : (wk > g.n ? wk - g.n : wk);
            if (g.interior(wi, wj, wk) && !mk.solid(g, wi, wj, wk)) w |= 1ull << (36 + q);
        }
    }
    links[t] = w;
}

// One warp per 32-bit mask word: lane b tests node i = 32w + b + 1 of the row and the
// ballot is the word.  Every lane of a warp shares the word, so the early return and
// the ballot are warp-uniform.
__global__ void k_voxelise(Geo g, VoxShape S, uint32_t* bits, int wpr) {
    const int64_t word = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (word >= (int64_t)g.m * g.n * wpr) return;
    const int64_t row = word / wpr;
    const int i = 32 * (int)(word % wpr) + lane + 1;
    const int64_t j = row % g.m + 1, k = row / g.m + 1;
    const bool solid = i <= g.l && vox_solid(S, (int64_t)i + S.off[0], j + S.off[1], k + S.off[2]);
    const uint32_t b = __ballot_sync(0xffffffffu, solid);
    if (lane == 0) bits[word] = b;
}

// out[0] solid voxels, out[1] of them on the column i = 1, out[2] on i = l (integer
// sums: the result does not depend on the order of the atomics).
__global__ void k_mask_counts(const uint32_t* bits, Geo g, int wpr, unsigned long long* out) {
    const int64_t words = (int64_t)g.m * g.n * wpr;
    const int wl = (g.l - 1) >> 5, bl = (g.l - 1) & 31;
    unsigned long long c[3] = {0, 0, 0};
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < words; t += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t v = bits[t];
        const int w = (int)(t % wpr);
        c[0] += __popc(v);
        if (w == 0) c[1] += v & 1u;
        if (w == wl) c[2] += (v >> bl) & 1u;
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        unsigned long long x = c[a];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0 && x) atomicAdd(out + a, x);
    }
}

struct IsSolid {
    Geo g;
    Mask mk;
    __device__ bool operator()(int32_t lin) const {
        const int i = (int)(lin % g.l) + 1, j = (int)((lin / g.l) % g.m) + 1, k = (int)(lin / g.lm) + 1;
        return mk.solid(g, i, j, k);
    }
};

// Fortran record [12][i][j][k][12] of each listed voxel (gfortran unformatted sequential).
__global__ void k_obs_records(Geo g, const int32_t* list, int64_t n, int32_t* rec) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int64_t lin = list[t];
    int32_t* r = rec + 5 * t;
    r[0] = 12;
    r[1] = (int32_t)(lin % g.l) + 1;
    r[2] = (int32_t)((lin / g.l) % g.m) + 1;
    r[3] = (int32_t)(lin / g.lm) + 1;
    r[4] = 12;
}

unsigned blocks_for(int64_t n, int tpb) { return (unsigned)((n + tpb - 1) / tpb); }

}  // namespace

void launch_voxelise(const Geo& g, const VoxShape& S, uint32_t* bits, int wpr, cudaStream_t st) {
    const int64_t threads = (int64_t)g.m * g.n * wpr * 32;
    k_voxelise<<<blocks_for(threads, 256), 256, 0, st>>>(g, S, bits, wpr);
}

void launch_mask_counts(const uint32_t* bits, const Geo& g, int wpr, unsigned long long* out, cudaStream_t st) {
    const int64_t words = (int64_t)g.m * g.n * wpr;
    const unsigned blocks = (unsigned)std::min<int64_t>(blocks_for(words, 256), 148 * 8);
    cudaMemsetAsync(out, 0, 3 * sizeof(unsigned long long), st);
    k_mask_counts<<<blocks, 256, 0, st>>>(bits, g, wpr, out);
}

cudaError_t obstacle_records(const Geo& g, const Mask& mk, int64_t nsolid, int32_t* rec, cudaStream_t st) {
    if (nsolid <= 0) return cudaSuccess;
    thrust::counting_iterator<int32_t> it(0);
    int32_t* list = nullptr;
    int* d_count = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    int h_count = 0;
    const IsSolid pred{g, mk};
    cudaError_t e = cub::DeviceSelect::If(nullptr, tmp_bytes, it, (int32_t*)nullptr, d_count, (int)g.N, pred, st);
    if (e == cudaSuccess) e = cudaMalloc(&tmp, tmp_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&d_count, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&list, sizeof(int32_t) * (size_t)nsolid);
    if (e == cudaSuccess) e = cub::DeviceSelect::If(tmp, tmp_bytes, it, list, d_count, (int)g.N, pred, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_count, d_count, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess && h_count != nsolid) e = cudaErrorInvalidValue;  // mask changed under us: cannot happen
    if (e == cudaSuccess) {
        k_obs_records<<<blocks_for(nsolid, 256), 256, 0, st>>>(g, list, nsolid, rec);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (tmp) cudaFree(tmp);
    if (d_count) cudaFree(d_count);
    if (list) cudaFree(list);
    return e;
}

void launch_build_mask(const int32_t* obs, const Geo& g, uint32_t* bits, int wpr, cudaStream_t st) {
    const int64_t words = (int64_t)g.m * g.n * wpr;
    k_build_mask<<<blocks_for(words, 256), 256, 0, st>>>(obs, g, bits, wpr);
}

void launch_flag_boundary_solid(const Geo& g, const Mask& mk, uint8_t* flags, cudaStream_t st) {
    k_flag_boundary_solid<<<blocks_for(g.N, 256), 256, 0, st>>>(g, mk, flags);
}

void launch_bsolid_links(const Geo& g, const Mask& mk, const int bc[6], const int32_t* list, int64_t n,
                         uint64_t* links, cudaStream_t st) {
    if (n <= 0) return;
    const int per_x = (bc[0] == 0 && bc[1] == 0), per_y = (bc[2] == 0 && bc[3] == 0);
    const int per_z = (bc[4] == 0 && bc[5] == 0);
    k_bsolid_links<<<blocks_for(n, 256), 256, 0, st>>>(g, mk, per_x, per_y, per_z, list, n, links);
}

void launch_links(const Geo& g, const Mask& mk, uint32_t* links, cudaStream_t st) {
    k_links<<<blocks_for(g.N, 256), 256, 0, st>>>(g, mk, links);
}

int64_t compact_flags(const uint8_t* flags, int64_t n, int32_t* out, cudaStream_t st, cudaError_t* err) {
    *err = cudaSuccess;
    thrust::counting_iterator<int32_t> it(0);
    int* d_count = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    int h_count = 0;
    cudaError_t e = cub::DeviceSelect::Flagged(nullptr, tmp_bytes, it, flags, out, d_count, (int)n, st);
    if (e == cudaSuccess) e = cudaMalloc(&tmp, tmp_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&d_count, sizeof(int));
    if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(tmp, tmp_bytes, it, flags, out, d_count, (int)n, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_count, d_count, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (tmp) cudaFree(tmp);
    if (d_count) cudaFree(d_count);
    *err = e;
    return e == cudaSuccess ? (int64_t)h_count : -1;
}

}  // namespace eup
