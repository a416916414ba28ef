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
    if (i == 1 || i == g.l) {
#pragma unroll
        for (int q = 0; q < 18; ++q) {
            const R v = stored_value<S, R>(x[q], q, dst.scale, dst.inv_scale);
            if (i == 1) dst.xface[xface_idx(g, 0, q, j, k)] = v;
            if (i == g.l) dst.xface[xface_idx(g, 1, q, j, k)] = v;
        }
    }
}

// ---------------------------------------------------------------------------
// Vectorised variant: each thread owns VW consecutive x-nodes of one (j,k)
// row, so every population moves as one 16-byte (or 8-byte) load and store.
// Pulls along x (cx = +-1) need one element of the neighbouring thread's
// vector: it comes from the adjacent lane by warp shuffle; lane 31/0 read it
// from global memory (an L2 hit: the neighbouring warp loads the same line),
// and the first/last thread of a row reads the x halo of the source row from
// the halo shell.  Rows on the y/z boundary planes pull through the shell
// node by node.  Requires l % (32*VW) == 0 and blockDim.x % 32 == 0, so a warp
// never spans two rows and every branch below is warp-uniform.
// ---------------------------------------------------------------------------
template <int BYTES> struct RawVec;
template <> struct RawVec<16> { using T = uint4; };
template <> struct RawVec<8> { using T = uint2; };

template <typename S, int VW>
struct Pack {
    using T = typename RawVec<sizeof(S) * VW>::T;
    union {
        T raw;
        S s[VW];
    };
};

template <typename S, int VW>
__device__ __forceinline__ void ld_pack(Pack<S, VW>& p, const S* ptr) {
    p.raw = __ldg(reinterpret_cast<const typename Pack<S, VW>::T*>(ptr));
}
template <typename S, int VW>
__device__ __forceinline__ void st_pack(S* ptr, const Pack<S, VW>& p) {
    *reinterpret_cast<typename Pack<S, VW>::T*>(ptr) = p.raw;
}

template <typename S, typename R, int VW>
__global__ void __launch_bounds__(256) k_stream_collide_vec(Lat<S, R> src, Lat<S, R> dst, Geo g, Phys<R> ph) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;  // vector index within the row
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z + 1;
    if (j > g.m) return;  // whole warps only
    const int nvec = g.l / VW;
    const int lane = threadIdx.x & 31;
    const int i0 = t * VW + 1;
    const int64_t row = (int64_t)(j - 1) * g.l + (int64_t)(k - 1) * g.lm;
    const bool face = (j == 1) | (j == g.m) | (k == 1) | (k == g.n);

    Pack<S, VW> in[19];
    R edge[19];  // x-neighbour element for cx = +1 (left) and cx = -1 (right) populations
    if (!face) {
#pragma unroll
        for (int q = 0; q < 18; ++q) {
            const S* rp = src.pop[q] + row - (int64_t)cy_of(q) * g.l - (int64_t)cz_of(q) * g.lm;
            ld_pack<S, VW>(in[q], rp + (int64_t)t * VW);
            if (cx_of(q) == 1) {
                R e = __shfl_up_sync(0xffffffffu, Store<S, R>::load(in[q].s[VW - 1], q, src.inv_scale), 1);
                if (t == 0) e = src.ghost[(int64_t)q * g.G + g.gidx(0, j - cy_of(q), k - cz_of(q))];
                else if (lane == 0) e = Store<S, R>::load(rp[(int64_t)t * VW - 1], q, src.inv_scale);
                edge[q] = e;
            } else if (cx_of(q) == -1) {
                R e = __shfl_down_sync(0xffffffffu, Store<S, R>::load(in[q].s[0], q, src.inv_scale), 1);
                if (t == nvec - 1) e = src.ghost[(int64_t)q * g.G + g.gidx(g.l + 1, j - cy_of(q), k - cz_of(q))];
                else if (lane == 31) e = Store<S, R>::load(rp[(int64_t)t * VW + VW], q, src.inv_scale);
                edge[q] = e;
            }
        }
        ld_pack<S, VW>(in[18], src.pop[18] + row + (int64_t)t * VW);
    }

    Pack<S, VW> out[19];
#pragma unroll
    for (int e = 0; e < VW; ++e) {
        R x[19];
        if (!face) {
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                const int c = (q == 18) ? 0 : cx_of(q);
                if (c == 0) x[q] = Store<S, R>::load(in[q].s[e], q, src.inv_scale);
                else if (c == 1) x[q] = (e == 0) ? edge[q] : Store<S, R>::load(in[q].s[e - 1], q, src.inv_scale);
                else x[q] = (e == VW - 1) ? edge[q] : Store<S, R>::load(in[q].s[e + 1], q, src.inv_scale);
            }
        } else {
            const int i = i0 + e;
#pragma unroll
            for (int q = 0; q < 18; ++q) x[q] = lat_load(src, g, q, i - cx_of(q), j - cy_of(q), k - cz_of(q));
            x[18] = Store<S, R>::load(src.pop[18][row + i - 1], 18, src.inv_scale);
        }
        collide<R>(x, ph.omega, ph.omega1, ph.fgrad);
#pragma unroll
        for (int q = 0; q < 19; ++q) out[q].s[e] = Store<S, R>::store(x[q], q, dst.scale);
        if ((e == 0 && t == 0) || (e == VW - 1 && t == nvec - 1)) {  // x = 1 or x = l column
            const int side = (e == 0 && t == 0) ? 0 : 1;
#pragma unroll
            for (int q = 0; q < 18; ++q)
                dst.xface[xface_idx(g, side, q, j, k)] = Store<S, R>::load(out[q].s[e], q, dst.inv_scale);
        }
    }
#pragma unroll
    for (int q = 0; q < 19; ++q) st_pack<S, VW>(dst.pop[q] + row + (int64_t)t * VW, out[q]);
}

template <typename S> struct VecWidth { static constexpr int value = 16 / sizeof(S); };

}  // namespace

template <typename S, typename R>
void launch_stream_collide(const Lat<S, R>& src, const Lat<S, R>& dst, const Geo& g, const Phys<R>& ph,
                           int variant, cudaStream_t st) {
    constexpr int VW = VecWidth<S>::value;
    const bool vec_ok = (g.l % (32 * VW)) == 0;
    if (!(variant & 1) && vec_ok) {
        const int nvec = g.l / VW;
        int tx = nvec;
        while (tx > 256) tx /= 2;  // nvec is a multiple of 32; keep tx a multiple of 32 dividing nvec
        if (tx % 32 != 0 || nvec % tx != 0) tx = 32;
        const int ty = (256 / tx) > 0 ? 256 / tx : 1;
        dim3 block(tx, ty, 1);
        dim3 grid(nvec / tx, (g.m + ty - 1) / ty, g.n);
        k_stream_collide_vec<S, R, VW><<<grid, block, 0, st>>>(src, dst, g, ph);
        return;
    }
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
