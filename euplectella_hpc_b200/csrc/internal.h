// Internal interfaces between the host entry points (abi.cu) and the CUDA
// kernels (k_bc.cu, k_step.cu, k_setup.cu).  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "lbm_common.cuh"

namespace eup {

// Bit-packed solid mask: one bit per interior node, rows along x padded to
// 32-bit words (wpr words per (j,k) row).
struct Mask {
    const uint32_t* bits;
    int wpr;
    __device__ __forceinline__ bool solid(const Geo& g, int i, int j, int k) const {
        if (bits == nullptr || !g.interior(i, j, k)) return false;
        const int64_t row = (int64_t)(j - 1) + (int64_t)g.m * (k - 1);
        return (bits[row * wpr + ((i - 1) >> 5)] >> ((i - 1) & 31)) & 1u;
    }
};

// Reduction scratch: per-block partial sums and a completion counter.  The
// last block to finish adds the partials in block order, so results do not
// depend on scheduling.
struct Reduce {
    double* partials;     // [max_blocks * width]
    unsigned int* counter;
    int max_blocks;
};

constexpr int kReduceMaxBlocks = 4096;
constexpr int kReduceWidth = 8;

// Halo-plane operations of CODE/SRC/bcond.bc.F90, launched in the reference's order;
// returns the number of kernels launched.
template <typename S, typename R>
int launch_bc(const Lat<S, R>& L, const Geo& g, const int bc[6], const Phys<R>& ph, cudaStream_t st);

// Bounce-back on solid voxels touching fluid/halo (CODE/SRC/bcond.obs.F90) and the
// FP64 momentum-exchange force of the state it reads, written to
// series[3*(*d_itime % cap)]; with `advance` the device step counter is incremented.
template <typename S, typename R>
void launch_bounce_drag(const Lat<S, R>& L, const Geo& g, const Mask& mk, const int bc[6],
                        const int32_t* list, int64_t nlist, bool do_bounce, const Reduce& red,
                        double* series, int64_t cap, int64_t* d_itime, bool advance, cudaStream_t st);

// x-face copy of the current lattice (needed once after an upload).
template <typename S, typename R>
void launch_fill_xface(const Lat<S, R>& L, const Geo& g, cudaStream_t st);

// Fused pull stream + collide (CODE/SRC/movef.F90 + CODE/SRC/col.F90): src -> dst.
template <typename S, typename R>
void launch_stream_collide(const Lat<S, R>& src, const Lat<S, R>& dst, const Geo& g,
                           const Phys<R>& ph, int variant, cudaStream_t st);

// FP64 sums of CODE/SRC/diagno.F90 into out[5] (device pointer).
template <typename S, typename R>
void launch_monitor(const Lat<S, R>& L, const Geo& g, const Mask& mk, const Reduce& red,
                    double* out, cudaStream_t st);

// rho,u at given nodes into out[4*npts] (device pointers).
template <typename S, typename R>
void launch_probes(const Lat<S, R>& L, const Geo& g, int npts, const int32_t* ijk, double* out,
                   cudaStream_t st);

// Scatter one haloed host-layout array (T) into lattice population q + shell.
template <typename S, typename R, typename T>
void launch_scatter(const Lat<S, R>& L, const Geo& g, int q, const T* staging, cudaStream_t st);
template <typename S, typename R, typename T>
void launch_gather(const Lat<S, R>& L, const Geo& g, int q, T* staging, cudaStream_t st);

// Set-up kernels (k_setup.cu).
void launch_build_mask(const int32_t* obs, const Geo& g, uint32_t* bits, int wpr, cudaStream_t st);
void launch_flag_boundary_solid(const Geo& g, const Mask& mk, uint8_t* flags, cudaStream_t st);
void launch_links(const Geo& g, const Mask& mk, uint32_t* links, cudaStream_t st);
// Ordered compaction of flagged linear indices; returns the count (synchronous).
int64_t compact_flags(const uint8_t* flags, int64_t n, int32_t* out, cudaStream_t st, cudaError_t* err);

}  // namespace eup
