// Fused pull stream + collide: for every interior node x,
//   f_q = a_q(x - c_q)            (CODE/SRC/movef.F90:48-65; a19 stays, :125 of col)
//   a'  = collide(f)              (CODE/SRC/col.F90:127-229)
// reading the source lattice and halo shell, writing the destination lattice.
// Nodes whose 18 upstream neighbours are all interior take the fast path
// (plain shifted loads); nodes on the six boundary planes resolve each pull
// through the halo shell.
#include "internal.h"

namespace eup {

namespace {

// One thread per node; grid (ceil(l/bx), m, n).
template <typename S, typename R>
__global__ void __launch_bounds__(128) k_stream_collide_scalar(Lat<S, R> src, Lat<S, R> dst, Geo g, Phys<R> ph) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y + 1;
    const int k = blockIdx.z + 1;
    if (i > g.l) return;
    const int64_t lin = g.lin(i, j, k);
    R x[19];
    const bool face = (i == 1) | (i == g.l) | (j == 1) | (j == g.m) | (k == 1) | (k == g.n);
    if (!face) {
#pragma unroll
        for (int q = 0; q < 18; ++q) {
            const int64_t s = lin - cx_of(q) - (int64_t)cy_of(q) * g.l - (int64_t)cz_of(q) * g.lm;
            x[q] = Store<S, R>::load(src.pop[q][s], q, src.inv_scale);
        }
    } else {
#pragma unroll
        for (int q = 0; q < 18; ++q) x[q] = lat_load(src, g, q, i - cx_of(q), j - cy_of(q), k - cz_of(q));
    }
    x[18] = Store<S, R>::load(src.pop[18][lin], 18, src.inv_scale);
    collide<R>(x, ph.omega, ph.omega1, ph.fgrad);
#pragma unroll
    for (int q = 0; q < 19; ++q) dst.pop[q][lin] = Store<S, R>::store(x[q], q, dst.scale);
}

}  // namespace

template <typename S, typename R>
void launch_stream_collide(const Lat<S, R>& src, const Lat<S, R>& dst, const Geo& g, const Phys<R>& ph,
                           int variant, cudaStream_t st) {
    (void)variant;
    const int bx = 128;
    dim3 grid((g.l + bx - 1) / bx, g.m, g.n);
    k_stream_collide_scalar<S, R><<<grid, bx, 0, st>>>(src, dst, g, ph);
}

template void launch_stream_collide<float, float>(const Lat<float, float>&, const Lat<float, float>&,
                                                  const Geo&, const Phys<float>&, int, cudaStream_t);
template void launch_stream_collide<double, double>(const Lat<double, double>&, const Lat<double, double>&,
                                                    const Geo&, const Phys<double>&, int, cudaStream_t);
template void launch_stream_collide<__half, float>(const Lat<__half, float>&, const Lat<__half, float>&,
                                                   const Geo&, const Phys<float>&, int, cudaStream_t);
template void launch_stream_collide<__nv_bfloat16, float>(const Lat<__nv_bfloat16, float>&,
                                                          const Lat<__nv_bfloat16, float>&, const Geo&,
                                                          const Phys<float>&, int, cudaStream_t);

}  // namespace eup
