// Internal interfaces between the host entry points (abi.cu) and the CUDA
// kernels (k_bc.cu, k_step.cu, k_setup.cu).  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

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

// ---- block reduction into deterministic per-block partials ----------------------------
template <int W>
__device__ __forceinline__ void block_reduce_store(double (&v)[W], const Reduce& red, double* out, double* series = nullptr,
                                   int64_t cap = 0, int64_t* d_itime = nullptr, int advance = 0,
                                   int slot_offset = 0) {
    __shared__ double sh[32][W];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < W; ++c)
        for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_down_sync(0xffffffffu, v[c], o);
    if (lane == 0)
        for (int c = 0; c < W; ++c) sh[warp][c] = v[c];
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        for (int c = 0; c < W; ++c) {
            double s = 0.0;
            for (int w = 0; w < nw; ++w) s += sh[w][c];
            red.partials[(int64_t)blockIdx.x * W + c] = s;
        }
        __threadfence();
        const unsigned done = atomicAdd(red.counter, 1u);
        last = (done == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the last block adds the partials: thread t takes blocks t, t+blockDim, ...
    // (independent loads, fixed assignment), then the same fixed tree as above
    double s[W];
#pragma unroll
    for (int c = 0; c < W; ++c) s[c] = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
        for (int c = 0; c < W; ++c) s[c] += __ldcg(red.partials + (int64_t)b * W + c);
#pragma unroll
    for (int c = 0; c < W; ++c)
        for (int o = 16; o > 0; o >>= 1) s[c] += __shfl_down_sync(0xffffffffu, s[c], o);
    __syncthreads();
    if (lane == 0)
        for (int c = 0; c < W; ++c) sh[warp][c] = s[c];
    __syncthreads();
    if (threadIdx.x == 0) {
        double* dst = out;
        if (series) {
            const int64_t t = *(volatile int64_t*)d_itime;
            dst = series + W * ((t + slot_offset) % cap);
            if (advance) *d_itime = t + 1;
        }
        const int nw = (blockDim.x + 31) >> 5;
        for (int c = 0; c < W; ++c) {
            double tot = 0.0;
            for (int w = 0; w < nw; ++w) tot += sh[w][c];
            dst[c] = tot;
        }
        *red.counter = 0u;
    }
}

// Halo-plane operations of CODE/SRC/bcond.bc.F90 in the reference's order; returns the
// number of kernels launched.  With `bar` (three zeroed words of device memory owned by the
// caller, used by one stream at a time) and a device where prepare_bc_fused found cooperative
// launches usable in CUDA graphs, all blocks run as phases of one launch separated by grid
// barriers (measured slower); otherwise, and by default, one launch per block.
template <typename S, typename R>
int launch_bc(const Lat<S, R>& L, const Geo& g, const int bc[6], const Phys<R>& ph, cudaStream_t st,
              unsigned int* bar = nullptr);
// Once per device (outside graph capture): occupancy of the single-launch halo kernel, and a
// cooperative launch captured into a graph and run once, using `bar` (left zeroed).
cudaError_t prepare_bc_fused(unsigned int* bar);

// Bounce-back on solid voxels touching fluid/halo (CODE/SRC/bcond.obs.F90) and the
// FP64 momentum-exchange force of the state it reads, written to
// series[3*(*d_itime % cap)]; with `advance` the device step counter is incremented.
// links[t] classifies the 18 neighbours of list[t] (see launch_bsolid_links).
template <typename S, typename R>
void launch_bounce_drag(const Lat<S, R>& L, const Geo& g, const int bc[6], const int32_t* list,
                        const uint64_t* links, int64_t nlist, bool do_bounce, const Reduce& red, double* series,
                        int64_t cap, int64_t* d_itime, bool advance, cudaStream_t st);

// x-slab faces: the five populations crossing an x face, (m+2)(n+2) values each.
template <typename S, typename R>
void launch_pack_x(const Lat<S, R>& L, const Geo& g, int side, R* out, cudaStream_t st);
template <typename S, typename R>
void launch_unpack_x(const Lat<S, R>& L, const Geo& g, int side, const R* in, cudaStream_t st);
template <typename S, typename R>
void launch_pack_x_rim(const Lat<S, R>& L, const Geo& g, int sides, cudaStream_t st);
template <typename S, typename R>
void launch_unpack_x_view(const Lat<S, R>& L, const Geo& g, int side, const R* in, cudaStream_t st);

// x-face copy of the current lattice (needed once after an upload).
template <typename S, typename R>
void launch_fill_xface(const Lat<S, R>& L, const Geo& g, cudaStream_t st);

// Fused pull stream + collide (CODE/SRC/movef.F90 + CODE/SRC/col.F90): src -> dst, over
// every node (kStreamAll), or split into the columns that do not pull from the x halo
// planes (kStreamInterior) and the two that do (kStreamFaces), so that an x-slab can
// receive its halo planes while the interior streams.
enum { kStreamAll = 0, kStreamInterior = 1, kStreamFaces = 2 };
// Kernel attributes the stream-collide launches need (once per device, outside graph capture).
cudaError_t prepare_stream_collide();
// Number of bounded waits of the staged stream-collide kernel that ran out on this device
// since the last call (each stopped its CTA's stores: the step's result is then incomplete);
// the count restarts from zero once read.
cudaError_t staged_wait_timeouts(unsigned int* count);
template <typename S, typename R>
void launch_stream_collide(const Lat<S, R>& src, const Lat<S, R>& dst, const Geo& g,
                           const Phys<R>& ph, int variant, cudaStream_t st, int part = kStreamAll);

// Reference-form diagnostics (CODE/SRC/prof_*.F90, varm.F90, flux_X/flux_Y.F90):
// a line of per-node u, w, v, den in R; per-plane means; the FP64 face sums of
// the control-volume stresses of box = {i1, i2, j1, j2, k1, k2} (already clipped).
template <typename S, typename R>
void launch_line(const Lat<S, R>& L, const Geo& g, int axis, int c1, int c2, double* out, cudaStream_t st);
template <typename S, typename R>
void launch_plane_means(const Lat<S, R>& L, const Geo& g, int axis, double* out, cudaStream_t st);
template <typename S, typename R>
void launch_cv_drag(const Lat<S, R>& L, const Geo& g, const int box[6], R omega, const Reduce& red, double* out,
                    cudaStream_t st);

// FP64 sums over the fluid nodes of a region (device byte mask, one per node) into out[6].
template <typename S, typename R>
void launch_region_sums(const Lat<S, R>& L, const Geo& g, const Mask& mk, const uint8_t* region, const Reduce& red,
                        double* out, cudaStream_t st);

// Population q of the seeded equilibrium initial state (init_eq.h) into a
// haloed staging array of (l+2)(m+2)(n+2) elements.
template <typename T>
void launch_init_population(T* staging, const Geo& g, int q, double u_in, double amp, uint64_t seed, cudaStream_t st);

// FP64 sums of CODE/SRC/diagno.F90 into out[5] (device pointer).
template <typename S, typename R>
void launch_monitor(const Lat<S, R>& L, const Geo& g, const Mask& mk, const Reduce& red,
                    double* out, cudaStream_t st);

// rho,u at given nodes into out[4*npts] (device pointers).
template <typename S, typename R>
void launch_probes(const Lat<S, R>& L, const Geo& g, int npts, const int32_t* ijk, double* out,
                   cudaStream_t st);

// Scatter one haloed host-layout array (T) into lattice population q + shell; a
// value that is not finite sets bit q of *bad (device pointer).
template <typename S, typename R, typename T>
void launch_scatter(const Lat<S, R>& L, const Geo& g, int q, const T* staging, unsigned int* bad, cudaStream_t st);
template <typename S, typename R, typename T>
void launch_gather(const Lat<S, R>& L, const Geo& g, int q, T* staging, cudaStream_t st);

// Set-up kernels (k_setup.cu).
void launch_build_mask(const int32_t* obs, const Geo& g, uint32_t* bits, int wpr, cudaStream_t st);
// Device voxeliser (geometry.h): the bit-packed mask of shape S.
struct VoxShape;
void launch_voxelise(const Geo& g, const VoxShape& S, uint32_t* bits, int wpr, cudaStream_t st);
// out[0..2] = solid voxels, solid voxels at i = 1, at i = l.
void launch_mask_counts(const uint32_t* bits, const Geo& g, int wpr, unsigned long long* out, cudaStream_t st);
// The nsolid solid voxels of the mask, i fastest, as Fortran records [12][i][j][k][12]
// (rec holds 5 nsolid int32); synchronises st.
cudaError_t obstacle_records(const Geo& g, const Mask& mk, int64_t nsolid, int32_t* rec, cudaStream_t st);
void launch_flag_boundary_solid(const Geo& g, const Mask& mk, uint8_t* flags, cudaStream_t st);
void launch_links(const Geo& g, const Mask& mk, uint32_t* links, cudaStream_t st);
// Neighbour classification of each boundary-solid voxel: bit q (0..17) neighbour
// x + c_q is interior fluid, bit 18+q it is a halo node, bit 36+q that halo node
// wraps across a periodic axis onto interior fluid.
void launch_bsolid_links(const Geo& g, const Mask& mk, const int bc[6], const int32_t* list, int64_t n,
                         uint64_t* links, cudaStream_t st);
// Ordered compaction of flagged linear indices; returns the count (synchronous).
int64_t compact_flags(const uint8_t* flags, int64_t n, int32_t* out, cudaStream_t st, cudaError_t* err);

// ---- partial bounce-back and its adjoint (k_adjoint.cu) -------------------------
// Where the adjoint of each halo value goes, derived on the host by running the
// reference's halo blocks on symbols.  copy_*: halo slots holding a copy of an
// interior population, grouped by source key q*N + lin (CSR: copy_start).
// out_*: halo slots holding an outflow equilibrium, grouped by the x = l node
// (j-1) + (k-1)*m they are computed from, with the population produced.
struct HaloAdjointTables {
    std::vector<int64_t> copy_key;
    std::vector<int32_t> copy_start;
    std::vector<int64_t> copy_slot;
    std::vector<int32_t> out_jk;
    std::vector<int32_t> out_start;
    std::vector<int64_t> out_slot;
    std::vector<int8_t> out_q;
};
struct HaloAdjointDevice {
    const int64_t* copy_key = nullptr;
    const int32_t* copy_start = nullptr;
    const int64_t* copy_slot = nullptr;
    int64_t ncopy = 0;
    const int32_t* out_jk = nullptr;
    const int32_t* out_start = nullptr;
    const int64_t* out_slot = nullptr;
    const int8_t* out_q = nullptr;
    int64_t nout = 0;
};
// Returns EUP_OK or EUP_ERR_UNSUPPORTED (err says why).
int build_halo_adjoint_tables(const Geo& g, const int bc[6], HaloAdjointTables* out, std::string* err);

// One partial-bounce-back step src -> dst (any storage; FP32 arithmetic for 16-bit storage):
// the plain stream-collide, then the mixing f* = (1 - n_s) BGK(f) + n_s f_opp on the ns_count
// voxels of ns_list (those with n_s > 0).  With `series` the FP64 force of the step goes to
// series[(itime + 1) % cap] and the device step counter advances; series == nullptr skips it
// (recomputation in the adjoint).
template <typename S, typename R>
void launch_pbb_step(const Lat<S, R>& src, const Lat<S, R>& dst, const Geo& g, const Phys<R>& ph, const R* ns,
                     const int32_t* ns_list, int64_t ns_count, const Reduce& red, double* series, int64_t cap,
                     int64_t* d_itime, cudaStream_t st);
// Adjoint of one partial-bounce-back step from state f (its halo shell holding the step's
// halo values); the adjoint fields lam are in the arithmetic type.  The adjoint is pushed:
// node x writes lam_out_q at the node x - c_q it pulled from, each slot once.  parts:
// kAdjInterior, the nodes 2..l-1 x 2..m-1 x 2..n-1, which read no halo value; kAdjFaces,
// the boundary-plane nodes (they read the step's halo values and write the halo part gmu);
// these two write disjoint slots and may run on different streams.  kAdjTransposes adds the
// halo adjoints back onto the interior slots they were copied from or computed from; it
// runs after both, since those slots may be ones the interior part writes.
enum { kAdjInterior = 1, kAdjFaces = 2, kAdjTransposes = 4, kAdjAll = 7 };
template <typename S, typename R>
void launch_pbb_adjoint(const Lat<S, R>& f, const Geo& g, const Phys<R>& ph, const R* ns, const Lat<R, R>& lam_in,
                        const Lat<R, R>& lam_out, R* gmu, double* grad, R gamma, const HaloAdjointDevice& t,
                        cudaStream_t st, int parts = kAdjAll);

}  // namespace eup
