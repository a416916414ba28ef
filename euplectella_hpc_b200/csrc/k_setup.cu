// Set-up kernels for the solid mask (CODE/SRC/build.obs.F90 feeds
// CODE/SRC/bcond.obs.F90): bit packing, link classification and the ordered
// list of solid voxels that touch fluid or halo.
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

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

unsigned blocks_for(int64_t n, int tpb) { return (unsigned)((n + tpb - 1) / tpb); }

}  // namespace

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
