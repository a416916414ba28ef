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

// What the kernels compute with: the population f itself (FP32/FP64 storage,
// reference arithmetic), or the scaled deviation D = (f - w)*S (16-bit
// storage, collide_dev).  Values from the halo shell are always f.
template <typename S, typename R>
struct KOps {
    static constexpr bool dev = DevStore<S>::value;
    static __device__ __forceinline__ R val(S raw, int q, const Lat<S, R>& L) {
        if constexpr (dev) return DevStore<S>::to_f(raw);
        else return Store<S, R>::load(raw, q, L.inv_scale);
    }
    static __device__ __forceinline__ R from_shell(R f, int q, const Lat<S, R>& L) {
        if constexpr (dev) return (f - weight<R>(q)) * L.scale;
        else return f;
    }
    static __device__ __forceinline__ R pull(const Lat<S, R>& L, const Geo& g, int q, int i, int j, int k) {
        if (g.interior(i, j, k)) return val(L.pop[q][g.lin(i, j, k)], q, L);
        return from_shell(L.ghost[(int64_t)q * g.G + g.gidx(i, j, k)], q, L);
    }
    static __device__ __forceinline__ void collide_node(R* x, const Phys<R>& ph, const Lat<S, R>& L) {
        if constexpr (dev) collide_dev(x, ph.omega, ph.omega1, ph.fgrad, L.scale, L.inv_scale);
        else collide<R>(x, ph.omega, ph.omega1, ph.fgrad);
    }
    static __device__ __forceinline__ S store(R v, int q, const Lat<S, R>& L) {
        if constexpr (dev) return DevStore<S>::from_f(v);
        else return Store<S, R>::store(v, q, L.scale);
    }
};

// Streamed populations of interior node (i, j, k); rowlin = l*((j-1) + m*(k-1))
// is the linear index of x = 1 on its row (32-bit: one lattice holds fewer than
// 2^31 nodes).  Every source row pointer depends on the row only, so it is the
// same for the whole warp and each load is that pointer plus the thread's x.
// Rows on the y/z boundary planes (warp-uniform) resolve every pull through
// the halo shell.  Elsewhere all 18 shifted loads are issued unconditionally --
// for such rows every shifted index stays inside [0, N): D3Q19 has no (1,1,1)
// diagonals, so x = 0 of row (j', k') is x = l of row (j'-1, k') with j' >= 1,
// k' >= 2 or j' >= 2 -- and the five x-halo values of the first/last node of a
// row replace them afterwards.
template <typename S, typename R>
__device__ __forceinline__ void gather_node(const Lat<S, R>& src, const Geo& g, int i, int j, int k, int rowlin,
                                            R (&x)[19]) {
    using K = KOps<S, R>;
    const int l = g.l, lm = (int)g.lm;
    const bool face_yz = (j == 1) | (j == g.m) | (k == 1) | (k == g.n);
    if (!face_yz) {
#pragma unroll
        for (int q = 0; q < 18; ++q) {
            const S* rp = src.pop[q] + (rowlin - cy_of(q) * l - cz_of(q) * lm);
            x[q] = K::val(rp[i - 1 - cx_of(q)], q, src);
        }
        if (i == 1) {
#pragma unroll
            for (int q = 0; q < 18; ++q)
                if (cx_of(q) == 1)
                    x[q] = K::from_shell(src.ghost[(int64_t)q * g.G + g.gidx(0, j - cy_of(q), k - cz_of(q))], q, src);
        }
        if (i == l) {
#pragma unroll
            for (int q = 0; q < 18; ++q)
                if (cx_of(q) == -1)
                    x[q] = K::from_shell(src.ghost[(int64_t)q * g.G + g.gidx(l + 1, j - cy_of(q), k - cz_of(q))], q,
                                         src);
        }
    } else {
#pragma unroll
        for (int q = 0; q < 18; ++q) x[q] = K::pull(src, g, q, i - cx_of(q), j - cy_of(q), k - cz_of(q));
    }
    x[18] = K::val(src.pop[18][rowlin + i - 1], 18, src);
}

template <typename S, typename R>
__device__ __forceinline__ void scatter_node(const Lat<S, R>& dst, const Geo& g, int i, int j, int k, int rowlin,
                                             const R (&x)[19]) {
    using K = KOps<S, R>;
    S out[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        out[q] = K::store(x[q], q, dst);
        (dst.pop[q] + rowlin)[i - 1] = out[q];
    }
    if (i == 1 || i == g.l) {
#pragma unroll
        for (int q = 0; q < 18; ++q) {
            const R v = Store<S, R>::load(out[q], q, dst.inv_scale);
            if (i == 1) dst.xface[xface_idx(g, 0, q, j, k)] = v;
            if (i == g.l) dst.xface[xface_idx(g, 1, q, j, k)] = v;
        }
    }
}

template <typename S, typename R>
__device__ __forceinline__ void node_step(const Lat<S, R>& src, const Lat<S, R>& dst, const Geo& g,
                                          const Phys<R>& ph, int i, int j, int k) {
    const int rowlin = g.l * ((j - 1) + g.m * (k - 1));
    R x[19];
    gather_node(src, g, i, j, k, rowlin, x);
    KOps<S, R>::collide_node(x, ph, src);
    scatter_node(dst, g, i, j, k, rowlin, x);
}

// One thread per node of the columns i0 .. i0+ni-1; grid (ceil(ni/bx), m, n).
template <typename S, typename R>
__global__ void __launch_bounds__(128) k_stream_collide_scalar(Lat<S, R> src, Lat<S, R> dst, Geo g, Phys<R> ph,
                                                               int i0, int ni) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ni) return;
    node_step(src, dst, g, ph, i0 + t, (int)blockIdx.y + 1, (int)blockIdx.z + 1);
}

// The columns i = 1 and i = l (the only ones that pull from the x halo planes): one thread
// per (side, j, k); sides = 1 when l == 1.
template <typename S, typename R>
__global__ void __launch_bounds__(128) k_stream_collide_scalar_faces(Lat<S, R> src, Lat<S, R> dst, Geo g,
                                                                     Phys<R> ph, int sides) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)sides * g.m * g.n) return;
    const int side = (int)(t % sides);
    const int64_t row = t / sides;
    node_step(src, dst, g, ph, side ? g.l : 1, (int)(row % g.m) + 1, (int)(row / g.m) + 1);
}

// ---------------------------------------------------------------------------
// Pair kernel (FP32 arithmetic, l even): one thread streams and collides the
// two x-adjacent nodes (i, i+1), i odd.  The collision runs once on F2 values
// -- the packed FP32 instructions of sm_100 (fma .f32x2), rounded per lane
// exactly as the scalar code -- so the FP32 instruction count per node halves
// and the results equal the one-node kernel's bit for bit.  FP32 storage: the
// pulls with cx = 0 and every store move both nodes as one aligned 8-byte
// access, pulls with cx = +-1 are two scalar loads.  16-bit storage shifts
// population q by cx_q elements in memory, so all 19 pulls are aligned 4-byte
// loads (two nodes in one register: twice the bytes in flight per register);
// the stores of the ten populations with cx = +-1 are then two scalar stores.
// grid (ceil(l/2 / 128), m, n).
// ---------------------------------------------------------------------------
template <typename S> struct Vec2;
template <> struct Vec2<float> {
    using T = float2;
    static __device__ __forceinline__ float2 unpack(float2 v) { return v; }
    static __device__ __forceinline__ float2 pack(float2 v) { return v; }
    static __device__ __forceinline__ float lo(float2 v) { return v.x; }
    static __device__ __forceinline__ float hi(float2 v) { return v.y; }
};
template <> struct Vec2<__half> {
    using T = __half2;
    static __device__ __forceinline__ float2 unpack(__half2 v) { return __half22float2(v); }
    static __device__ __forceinline__ __half2 pack(float2 v) { return __float22half2_rn(v); }
    static __device__ __forceinline__ __half lo(__half2 v) { return __low2half(v); }
    static __device__ __forceinline__ __half hi(__half2 v) { return __high2half(v); }
};
template <> struct Vec2<__nv_bfloat16> {
    using T = __nv_bfloat162;
    static __device__ __forceinline__ float2 unpack(__nv_bfloat162 v) { return __bfloat1622float2(v); }
    static __device__ __forceinline__ __nv_bfloat162 pack(float2 v) { return __float22bfloat162_rn(v); }
    static __device__ __forceinline__ __nv_bfloat16 lo(__nv_bfloat162 v) { return __low2bfloat16(v); }
    static __device__ __forceinline__ __nv_bfloat16 hi(__nv_bfloat162 v) { return __high2bfloat16(v); }
};

// The two nodes of a y/z boundary row (warp-uniform), one by one through the halo shell.
template <typename S>
__device__ __forceinline__ void pair_through_shell(const Lat<S, float>& src, const Lat<S, float>& dst, const Geo& g,
                                                   const Phys<float>& ph, int i, int j, int k, int rowlin) {
#pragma unroll 1
    for (int e = 0; e < 2; ++e) {
        float x[19];
        gather_node(src, g, i + e, j, k, rowlin, x);
        KOps<S, float>::collide_node(x, ph, src);
        scatter_node(dst, g, i + e, j, k, rowlin, x);
    }
}

// Population q's source pointer moved back by c_q: the pull a_q(x - c_q) of node index x
// (0-based, x = i-1 + l (j-1 + m (k-1))) is base[q][x].  Set on the host per launch.
template <typename S>
struct PullBase {
    const S* p[19];
};

// lattice velocity components with the rest population (q = 18) as zero
__host__ __device__ constexpr int cx_of_or0(int q) { return q == 18 ? 0 : cx_of(q); }
__host__ __device__ constexpr int cy_of_or0(int q) { return q == 18 ? 0 : cy_of(q); }
__host__ __device__ constexpr int cz_of_or0(int q) { return q == 18 ? 0 : cz_of(q); }

// 16-bit storage: the 19 pulls of the pair (i, i+1) of an interior row as raw words
// (aligned in the shifted layout whatever cx is): one index for all of them.
template <typename S>
__device__ __forceinline__ void load_pair_raw(const PullBase<S>& pb, int i, int rowlin,
                                              typename Vec2<S>::T (&r)[19]) {
    using T2 = typename Vec2<S>::T;
    const uint32_t x = (uint32_t)(rowlin + i - 1);
#pragma unroll
    for (int q = 0; q < 19; ++q) r[q] = *reinterpret_cast<const T2*>(pb.p[q] + x);
}

// Everything after the pulls of an interior pair: the x-halo values of the first and
// last node of the row, the collision of both nodes as packed FP32, the x-face copy and
// the stores.
template <typename S>
__device__ __forceinline__ void finish_pair(const Lat<S, float>& src, const Lat<S, float>& dst, const Geo& g,
                                            const Phys<float>& ph, int i, int j, int k, int rowlin, F2 (&x)[19]) {
    using K = KOps<S, float>;
    using V2 = Vec2<S>;
    using T2 = typename V2::T;
    constexpr bool dev = DevStore<S>::value;
    const int l = g.l;
    if (i == 1) {
#pragma unroll
        for (int q = 0; q < 18; ++q)
            if (cx_of(q) == 1)
                x[q].v.x = K::from_shell(src.ghost[(int64_t)q * g.G + g.gidx(0, j - cy_of(q), k - cz_of(q))], q, src);
    }
    if (i + 1 == l) {
#pragma unroll
        for (int q = 0; q < 18; ++q)
            if (cx_of(q) == -1)
                x[q].v.y =
                    K::from_shell(src.ghost[(int64_t)q * g.G + g.gidx(l + 1, j - cy_of(q), k - cz_of(q))], q, src);
    }
    if constexpr (dev) collide_dev<F2>(x, ph.omega, ph.omega1, ph.fgrad, src.scale, src.inv_scale);
    else collide<F2>(x, F2(ph.omega), F2(ph.omega1), F2(ph.fgrad));
    if ((i == 1) | (i + 1 == l)) {  // x-face copy of the first/last column: the value a later load returns
#pragma unroll
        for (int q = 0; q < 18; ++q) {
            const T2 o = V2::pack(x[q].v);
            if (i == 1) dst.xface[xface_idx(g, 0, q, j, k)] = Store<S, float>::load(V2::lo(o), q, dst.inv_scale);
            if (i + 1 == l) dst.xface[xface_idx(g, 1, q, j, k)] = Store<S, float>::load(V2::hi(o), q, dst.inv_scale);
        }
    }
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        const T2 o = V2::pack(x[q].v);
        S* op = dst.pop[q] + rowlin + (i - 1);
        if (!dev || q == 18 || cx_of(q) == 0) {
            *reinterpret_cast<T2*>(op) = o;
        } else {  // odd address in the shifted layout
            op[0] = V2::lo(o);
            op[1] = V2::hi(o);
        }
    }
}

// The pair (i, i+1) of row (j, k).  Rows on the y/z boundary planes go node by node
// through the halo shell (warp-uniform in the row kernel, where a block is one row).
template <typename S>
__device__ __forceinline__ void pair_step(const Lat<S, float>& src, const Lat<S, float>& dst, const Geo& g,
                                          const Phys<float>& ph, const PullBase<S>& pb, int i, int j, int k) {
    using K = KOps<S, float>;
    using V2 = Vec2<S>;
    using T2 = typename V2::T;
    constexpr bool dev = DevStore<S>::value;
    const int l = g.l, lm = (int)g.lm;
    const int rowlin = l * ((j - 1) + g.m * (k - 1));
    const bool face_yz = (j == 1) | (j == g.m) | (k == 1) | (k == g.n);
    if (face_yz) {
        pair_through_shell(src, dst, g, ph, i, j, k, rowlin);
        return;
    }
    F2 x[19];
    if constexpr (dev) {
        T2 r[19];
        load_pair_raw(pb, i, rowlin, r);
#pragma unroll
        for (int q = 0; q < 19; ++q) x[q] = F2(V2::unpack(r[q]));
    } else {
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const int cx = (q == 18) ? 0 : cx_of(q), cy = (q == 18) ? 0 : cy_of(q), cz = (q == 18) ? 0 : cz_of(q);
            const S* rp = src.pop[q] + (rowlin - cy * l - cz * lm);
            if (cx == 0) {
                const float2 v = V2::unpack(*reinterpret_cast<const T2*>(rp + (i - 1)));
                x[q] = F2(K::val(v.x, q, src), K::val(v.y, q, src));
            } else {
                // both shifted loads are in bounds (interior rows; see gather_node)
                x[q] = F2(K::val(rp[i - 1 - cx], q, src), K::val(rp[i - cx], q, src));
            }
        }
    }
    finish_pair(src, dst, g, ph, i, j, k, rowlin, x);
}

// Pairs p0 .. p0+np-1 of every row (pair p: nodes 2p+1, 2p+2); grid (ceil(np/128), m, n).
template <typename S, int MINB>
__global__ void __launch_bounds__(128, MINB) k_stream_collide_pair(Lat<S, float> src, Lat<S, float> dst, Geo g,
                                                                   Phys<float> ph, PullBase<S> pb, int p0, int np) {
    const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (t >= np) return;
    pair_step(src, dst, g, ph, pb, 2 * (p0 + t) + 1, (int)blockIdx.y + 1, (int)blockIdx.z + 1);
}

// The first and last pair of every row (the only ones that pull from the x halo planes):
// one thread per (side, j, k); sides = 1 when l == 2.
template <typename S>
__global__ void __launch_bounds__(128, 6) k_stream_collide_pair_faces(Lat<S, float> src, Lat<S, float> dst, Geo g,
                                                                      Phys<float> ph, PullBase<S> pb, int sides) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)sides * g.m * g.n) return;
    const int side = (int)(t % sides);
    const int64_t row = t / sides;
    pair_step(src, dst, g, ph, pb, side ? g.l - 1 : 1, (int)(row % g.m) + 1, (int)(row / g.m) + 1);
}

template <typename S, typename R>
bool launch_pair(const Lat<S, R>& src, const Lat<S, R>& dst, const Geo& g, const Phys<R>& ph, int occ, int part,
                 cudaStream_t st) {
    if constexpr (sizeof(R) != 4) {
        return false;
    } else {
        if (g.l % 2 != 0) return false;
        // pair accesses: FP32 at the node's own address, 16-bit storage at the address
        // shifted back by cx_q (and its stores of cx = 0 populations)
        constexpr bool dev = DevStore<S>::value;
        for (int q = 0; q < Q; ++q) {
            const int cx = (q == 18) ? 0 : cx_of(q);
            const S* s0 = dev ? src.pop[q] - cx : src.pop[q];
            if (reinterpret_cast<uintptr_t>(s0) % (2 * sizeof(S)) != 0) return false;
            if ((!dev || cx == 0) && reinterpret_cast<uintptr_t>(dst.pop[q]) % (2 * sizeof(S)) != 0) return false;
        }
        // blocks of at most 128 threads, the row's pairs split evenly over its blocks (a
        // warp multiple), so short rows leave no idle threads (l = 192: one block of 96)
        const int npr = part == kStreamInterior ? g.l / 2 - 2 : (part == kStreamFaces ? 0 : g.l / 2);
        const int nblk = npr > 0 ? (npr + 127) / 128 : 1;
        const int bx = npr > 0 ? ((npr + nblk - 1) / nblk + 31) / 32 * 32 : 128;
        PullBase<S> pb;
        for (int q = 0; q < Q; ++q) {
            const int64_t c = (q == 18) ? 0 : (int64_t)cy_of(q) * g.l + (int64_t)cz_of(q) * g.lm + cx_of(q);
            pb.p[q] = src.pop[q] - c;  // only ever indexed at x >= c: the pull lies in the population
        }
        if (part == kStreamFaces) {
            const int sides = g.l == 2 ? 1 : 2;
            const int64_t threads = (int64_t)sides * g.m * g.n;
            k_stream_collide_pair_faces<S><<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(src, dst, g, ph, pb,
                                                                                             sides);
            return true;
        }
        // all pairs, or all but the first and last of each row
        const int p0 = part == kStreamInterior ? 1 : 0;
        const int np = part == kStreamInterior ? g.l / 2 - 2 : g.l / 2;
        if (np <= 0) return true;
        dim3 grid((np + bx - 1) / bx, g.m, g.n);
        // resident blocks of 128 threads per SM the register budget is sized for: by default
        // 6 (80 registers) for FP32 storage, 8 (64) for 16-bit storage, whose loads need fewer
        const int minb = occ > 0 ? occ + 3 : (sizeof(S) == 4 ? 6 : 8);
        switch (minb) {
            case 4: k_stream_collide_pair<S, 4><<<grid, bx, 0, st>>>(src, dst, g, ph, pb, p0, np); break;
            case 5: k_stream_collide_pair<S, 5><<<grid, bx, 0, st>>>(src, dst, g, ph, pb, p0, np); break;
            case 6: k_stream_collide_pair<S, 6><<<grid, bx, 0, st>>>(src, dst, g, ph, pb, p0, np); break;
            case 7: k_stream_collide_pair<S, 7><<<grid, bx, 0, st>>>(src, dst, g, ph, pb, p0, np); break;
            default: k_stream_collide_pair<S, 8><<<grid, bx, 0, st>>>(src, dst, g, ph, pb, p0, np); break;
        }
        return true;
    }
}

// ---------------------------------------------------------------------------
// Staged pair kernel (16-bit storage, l a multiple of 8).  The pulls of the interior rows
// (2 <= j <= m-1, 2 <= k <= n-1) come into shared memory by bulk asynchronous copies
// instead of per-thread loads.  In the x-shifted layout the pulls of population q for a
// run of consecutive nodes x0 .. x0+len-1 of one plane's interior rows are the run
// pb.p[q][x0 .. x0+len-1]: contiguous and, with x0 and len multiples of 8, 16-byte
// aligned.  A tile is kTileNodes such nodes (19 bulk copies).
//
// Persistent CTAs, warp-specialised: one producer warp and kConsumerWarps consumer warps
// (one pair of nodes per consumer thread and tile) share a ring of S stages, each with a
// "full" mbarrier (armed by the producer with the tile's byte count, completed by the
// copies) and an "empty" mbarrier (one arrival per consumer warp once the warp has read
// its words of the stage).  Consumers never wait for one another: a warp reads its 19
// words, releases the stage, then collides and stores while later tiles stream in.  The
// collision and stores are the register-pull kernel's (finish_pair: same arithmetic, same
// bits).  Rows on the y/z boundary planes, which pull through the halo shell, follow the
// tiles in the same launch, node by node.
//
// Every wait is bounded (2 s of the global timer).  A wait that runs out counts itself in
// g_staged_timeouts and stops its CTA: the consumers stop storing, the producer stops
// issuing and waits (bounded) for the copies it has in flight before the CTA returns.
// ---------------------------------------------------------------------------
__device__ unsigned int g_staged_timeouts;

constexpr int kStagedMaxStages = 4;
constexpr int kConsumerWarps = 8;
constexpr int kTileNodes = 64 * kConsumerWarps;       // 512 nodes, 256 pairs
constexpr int kStagedThreads = 32 * (kConsumerWarps + 1);
constexpr uint64_t kStagedWaitNs = 2000000000ull;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arm(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// true when the phase with this parity completed, false after kStagedWaitNs
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    if (mbar_test(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_test(bar, parity))
        if (global_ns() - t0 > kStagedWaitNs) return false;
    return true;
}
// bytes (a multiple of 16) from global src (16-byte aligned) to shared dst (16-byte aligned),
// completion counted on bar
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

struct StagedPlan {
    int plane_nodes;      // l * (m - 2): the interior rows of one plane
    int tiles_per_plane;  // ceil(plane_nodes / kTileNodes)
    int ntiles;           // tiles_per_plane * (n - 2)
    int nface;            // rows on the y/z boundary planes
    int stages;
    float inv_l;          // 1/l (rows of a node offset, corrected to exact)
};

template <typename S, int MINB>
__global__ void __launch_bounds__(kStagedThreads, MINB) k_stream_collide_staged(Lat<S, float> src, Lat<S, float> dst,
                                                                              Geo g, Phys<float> ph, PullBase<S> pb,
                                                                              StagedPlan sp) {
    using V2 = Vec2<S>;
    using T2 = typename V2::T;
    constexpr uint32_t kRunBytes = kTileNodes * sizeof(S);   // one population's run in a full tile
    constexpr uint32_t kStageBytes = 19 * kRunBytes;
    extern __shared__ __align__(128) unsigned char stage_mem[];
    __shared__ uint64_t full[kStagedMaxStages], empty[kStagedMaxStages];
    __shared__ int abort_flag;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int l = g.l, m = g.m;
    if (tid == 0) {
        for (int s = 0; s < sp.stages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kConsumerWarps);
        }
        mbar_init_fence();
        abort_flag = 0;
    }
    __syncthreads();

    // tile t: nodes x0 .. x0+len-1 (a multiple of 8 of them) of plane k's interior rows,
    // starting `off` nodes after the plane's row j = 2
    auto tile = [&](int t, int* k, int* off) {
        *k = 2 + t / sp.tiles_per_plane;
        *off = (t % sp.tiles_per_plane) * kTileNodes;
        return min(kTileNodes, sp.plane_nodes - *off);
    };
    const int first = blockIdx.x, stride = gridDim.x;
    if (warp == kConsumerWarps) {
        // producer: lane 0 arms each stage and issues its 19 copies once the consumers
        // have released it
        if (lane == 0) {
            int it = 0;
            for (int t = first; t < sp.ntiles; t += stride, ++it) {
                const int slot = it % sp.stages;
                if (it >= sp.stages && !mbar_wait_bounded(&empty[slot], (uint32_t)(it / sp.stages - 1) & 1u)) {
                    abort_flag = 1;
                    break;
                }
                if (abort_flag) break;
                int k, off;
                const int len = tile(t, &k, &off);
                const uint32_t bytes = (uint32_t)len * (uint32_t)sizeof(S);
                const uint32_t x0 = (uint32_t)l * (uint32_t)(1 + m * (k - 1)) + (uint32_t)off;
                unsigned char* base = stage_mem + (size_t)slot * kStageBytes;
                mbar_arm(&full[slot], 19u * bytes);
#pragma unroll 1
                for (int q = 0; q < 19; ++q) bulk_copy_g2s(base + q * kRunBytes, pb.p[q] + x0, bytes, &full[slot]);
            }
            // whatever is still in flight lands before the CTA's shared memory is released
            const int issued = it;
            for (int u = max(0, issued - sp.stages); u < issued; ++u)
                mbar_wait_bounded(&full[u % sp.stages], (uint32_t)(u / sp.stages) & 1u);
        }
    } else {
        int it = 0;
        const int c = tid;  // consumer thread: pair c of every tile
        for (int t = first; t < sp.ntiles; t += stride, ++it) {
            const int slot = it % sp.stages;
            if (!mbar_wait_bounded(&full[slot], (uint32_t)(it / sp.stages) & 1u)) {
                abort_flag = 1;
                break;
            }
            int k, off;
            const int len = tile(t, &k, &off);
            const unsigned char* base = stage_mem + (size_t)slot * kStageBytes;
            const bool active = 2 * c < len;
            F2 x[19];
            if (active) {
#pragma unroll
                for (int q = 0; q < 19; ++q)
                    x[q] = F2(V2::unpack(reinterpret_cast<const T2*>(base + q * kRunBytes)[c]));
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[slot]);
            if (abort_flag) break;
            if (active) {
                // node offset within the plane's interior rows -> row and column
                const int xr = off + 2 * c;
                int jr = __float2int_rz((float)xr * sp.inv_l);
                int ir = xr - jr * l;
                if (ir < 0) { --jr; ir += l; }
                if (ir >= l) { ++jr; ir -= l; }
                const int j = 2 + jr;
                finish_pair(src, dst, g, ph, ir + 1, j, k, l * ((j - 1) + m * (k - 1)), x);
            }
        }
    }
    __syncthreads();
    if (abort_flag) {
        if (tid == 0) atomicAdd(&g_staged_timeouts, 1u);
        return;
    }
    // rows on the y/z boundary planes: every pull through the halo shell
    const int half_l = l / 2;
    for (int f = blockIdx.x; f < sp.nface; f += stride) {
        int j, k;
        face_row(g, f, &j, &k);
        for (int p = tid; p < half_l; p += kStagedThreads) pair_step(src, dst, g, ph, pb, 2 * p + 1, j, k);
    }
}

constexpr int kStagedSmemLimit = 200 * 1024;   // dynamic shared memory the staged kernels opt into
constexpr int kSmemPerSM = 228 * 1024;

template <typename S>
bool launch_staged(const Lat<S, float>& src, const Lat<S, float>& dst, const Geo& g, const Phys<float>& ph,
                   int per_sm, cudaStream_t st) {
    if (g.l % 8 != 0 || g.l < 8) return false;
    StagedPlan sp;
    const int64_t plane_nodes = (int64_t)g.l * (g.m - 2);
    sp.plane_nodes = plane_nodes > 0 ? (int)plane_nodes : 0;
    sp.tiles_per_plane = (sp.plane_nodes + kTileNodes - 1) / kTileNodes;
    sp.ntiles = (g.n >= 3 && sp.plane_nodes > 0) ? sp.tiles_per_plane * (g.n - 2) : 0;
    const int nz = g.n >= 2 ? 2 : 1, ny = g.m >= 2 ? 2 : 1;
    sp.nface = nz * g.m + (g.n > 2 ? (g.n - 2) * ny : 0);
    sp.inv_l = 1.0f / (float)g.l;
    const int stage_bytes = 19 * kTileNodes * (int)sizeof(S);
    // per_sm CTAs per SM (3: 72 registers, 2: no spills), each with as many stages as fit
    sp.stages = kStagedMaxStages;
    while (sp.stages > 2 && per_sm * (stage_bytes * sp.stages + 1024) > kSmemPerSM) --sp.stages;
    // every run starts on a 16-byte boundary: the pull bases (a tile starts at a multiple of 8)
    PullBase<S> pb;
    for (int q = 0; q < Q; ++q) {
        pb.p[q] = src.pop[q] - (cy_of_or0(q) * (int64_t)g.l + cz_of_or0(q) * g.lm + cx_of_or0(q));
        if (reinterpret_cast<uintptr_t>(pb.p[q]) % 16 != 0) return false;
    }
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return false;
    const size_t smem = (size_t)stage_bytes * sp.stages;
    if (per_sm == 2)
        k_stream_collide_staged<S, 2><<<(unsigned)(2 * sms), kStagedThreads, smem, st>>>(src, dst, g, ph, pb, sp);
    else
        k_stream_collide_staged<S, 3><<<(unsigned)(3 * sms), kStagedThreads, smem, st>>>(src, dst, g, ph, pb, sp);
    return true;
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
    using K = KOps<S, R>;
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
        // 1) every vector load of the node group first, so all 19 are in flight together
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const int cy = (q == 18) ? 0 : cy_of(q), cz = (q == 18) ? 0 : cz_of(q);
            ld_pack<S, VW>(in[q], src.pop[q] + row - (int64_t)cy * g.l - (int64_t)cz * g.lm + (int64_t)t * VW);
        }
        // 2) the edge elements this lane cannot get from a neighbour lane: predicated
        //    loads from the row (lanes 0/31) or from the x halo (row ends)
        const bool lo_row = (t == 0), hi_row = (t == nvec - 1);
        const bool lo_glob = (lane == 0) && !lo_row, hi_glob = (lane == 31) && !hi_row;
#pragma unroll
        for (int q = 0; q < 18; ++q) {
            if (cx_of(q) == 0) continue;
            const S* rp = src.pop[q] + row - (int64_t)cy_of(q) * g.l - (int64_t)cz_of(q) * g.lm;
            R e = R(0);
            if (cx_of(q) == 1) {
                if (lo_glob) e = K::val(__ldg(rp + (int64_t)t * VW - 1), q, src);
                if (lo_row) e = K::from_shell(src.ghost[(int64_t)q * g.G + g.gidx(0, j - cy_of(q), k - cz_of(q))], q, src);
            } else {
                if (hi_glob) e = K::val(__ldg(rp + (int64_t)t * VW + VW), q, src);
                if (hi_row)
                    e = K::from_shell(src.ghost[(int64_t)q * g.G + g.gidx(g.l + 1, j - cy_of(q), k - cz_of(q))], q, src);
            }
            edge[q] = e;
        }
        // 3) neighbour-lane elements by shuffle
#pragma unroll
        for (int q = 0; q < 18; ++q) {
            if (cx_of(q) == 1) {
                const R e = __shfl_up_sync(0xffffffffu, K::val(in[q].s[VW - 1], q, src), 1);
                if (!lo_glob && !lo_row) edge[q] = e;
            } else if (cx_of(q) == -1) {
                const R e = __shfl_down_sync(0xffffffffu, K::val(in[q].s[0], q, src), 1);
                if (!hi_glob && !hi_row) edge[q] = e;
            }
        }
    }

    Pack<S, VW> out[19];
#pragma unroll
    for (int e = 0; e < VW; ++e) {
        R x[19];
        if (!face) {
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                const int c = (q == 18) ? 0 : cx_of(q);
                if (c == 0) x[q] = K::val(in[q].s[e], q, src);
                else if (c == 1) x[q] = (e == 0) ? edge[q] : K::val(in[q].s[e - 1], q, src);
                else x[q] = (e == VW - 1) ? edge[q] : K::val(in[q].s[e + 1], q, src);
            }
        } else {
            const int i = i0 + e;
#pragma unroll
            for (int q = 0; q < 18; ++q) x[q] = K::pull(src, g, q, i - cx_of(q), j - cy_of(q), k - cz_of(q));
            x[18] = K::val(src.pop[18][row + i - 1], 18, src);
        }
        K::collide_node(x, ph, src);
#pragma unroll
        for (int q = 0; q < 19; ++q) out[q].s[e] = K::store(x[q], q, dst);
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

// Nodes per thread of the vector kernels: 16-byte vectors (4 FP32, 2 FP64,
// 8 FP16/BF16) or 8-byte vectors (half that).
template <typename S> struct VecWidth { static constexpr int value = 16 / sizeof(S); };

template <typename S, typename R, int VW>
bool launch_vec(const Lat<S, R>& src, const Lat<S, R>& dst, const Geo& g, const Phys<R>& ph, cudaStream_t st) {
    if (g.l % (32 * VW) != 0) return false;
    for (int q = 0; q < Q; ++q)  // every row must start on a vector boundary
        if (reinterpret_cast<uintptr_t>(src.pop[q]) % (sizeof(S) * VW) != 0 ||
            reinterpret_cast<uintptr_t>(dst.pop[q]) % (sizeof(S) * VW) != 0)
            return false;
    const int nvec = g.l / VW;
    int tx = nvec;
    while (tx > 256) tx /= 2;  // nvec is a multiple of 32; keep tx a multiple of 32 dividing nvec
    if (tx % 32 != 0 || nvec % tx != 0) tx = 32;
    const int ty = (256 / tx) > 0 ? 256 / tx : 1;
    dim3 block(tx, ty, 1);
    dim3 grid(nvec / tx, (g.m + ty - 1) / ty, g.n);
    k_stream_collide_vec<S, R, VW><<<grid, block, 0, st>>>(src, dst, g, ph);
    return true;
}

}  // namespace

template <typename S, typename R>
void launch_stream_collide(const Lat<S, R>& src, const Lat<S, R>& dst, const Geo& g, const Phys<R>& ph,
                           int variant, cudaStream_t st, int part) {
    // EUP_STEP_VARIANT bit 0: 16-byte vectors, bit 2: 8-byte vectors (when l allows), bit 3: one
    // node per thread, bits 4-6: occupancy target of the two-node kernel (n + 3 blocks per SM),
    // bit 7: 16-bit storage staged in shared memory by bulk copies (l a multiple of 8; with
    // bit 11 two CTAs per SM instead of three); default: two nodes per thread (FP32
    // arithmetic, l even), the pulls loaded into registers.  (Bit 12 concerns the halo
    // kernels: all blocks in one cooperative launch instead of one launch per block.)  A split step (interior columns,
    // then the two x-face columns) uses the two-node or the one-node kernel.
    constexpr int VW = VecWidth<S>::value;
    if (part == kStreamAll) {
        if ((variant & 1) && launch_vec<S, R, VW>(src, dst, g, ph, st)) return;
        if ((variant & 4) && launch_vec<S, R, (VW / 2 > 0 ? VW / 2 : 1)>(src, dst, g, ph, st)) return;
        if constexpr (DevStore<S>::value) {  // opt-in: measured slower than the register pulls below
            if ((variant & 128) && !(variant & 8) && launch_staged<S>(src, dst, g, ph, (variant & 2048) ? 2 : 3, st))
                return;
        }
    }
    if (!(variant & 8) && launch_pair<S, R>(src, dst, g, ph, (variant >> 4) & 7, part, st)) return;
    const int bx = 128;
    if (part == kStreamFaces) {
        const int sides = g.l == 1 ? 1 : 2;
        const int64_t threads = (int64_t)sides * g.m * g.n;
        k_stream_collide_scalar_faces<S, R><<<(unsigned)((threads + bx - 1) / bx), bx, 0, st>>>(src, dst, g, ph, sides);
        return;
    }
    const int i0 = part == kStreamInterior ? 2 : 1;
    const int ni = part == kStreamInterior ? g.l - 2 : g.l;
    if (ni <= 0) return;
    dim3 grid((ni + bx - 1) / bx, g.m, g.n);
    k_stream_collide_scalar<S, R><<<grid, bx, 0, st>>>(src, dst, g, ph, i0, ni);
}

template void launch_stream_collide<float, float>(const Lat<float, float>&, const Lat<float, float>&,
                                                  const Geo&, const Phys<float>&, int, cudaStream_t, int);
template void launch_stream_collide<double, double>(const Lat<double, double>&, const Lat<double, double>&,
                                                    const Geo&, const Phys<double>&, int, cudaStream_t, int);
template void launch_stream_collide<__half, float>(const Lat<__half, float>&, const Lat<__half, float>&,
                                                   const Geo&, const Phys<float>&, int, cudaStream_t, int);
template void launch_stream_collide<__nv_bfloat16, float>(const Lat<__nv_bfloat16, float>&,
                                                          const Lat<__nv_bfloat16, float>&, const Geo&,
                                                          const Phys<float>&, int, cudaStream_t, int);

cudaError_t prepare_stream_collide() {
    // the staged kernels opt into more than 48 KB of dynamic shared memory (set once per
    // device, before any launch is captured into a graph)
    cudaError_t e = cudaSuccess;
    const void* ks[] = {(const void*)k_stream_collide_staged<__half, 2>, (const void*)k_stream_collide_staged<__half, 3>,
                        (const void*)k_stream_collide_staged<__nv_bfloat16, 2>,
                        (const void*)k_stream_collide_staged<__nv_bfloat16, 3>};
    for (const void* k : ks)
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kStagedSmemLimit);
    return e;
}

cudaError_t staged_wait_timeouts(unsigned int* count) {
    cudaError_t e = cudaMemcpyFromSymbol(count, g_staged_timeouts, sizeof(unsigned int));
    if (e == cudaSuccess && *count != 0) {  // reported once
        const unsigned int zero = 0;
        e = cudaMemcpyToSymbol(g_staged_timeouts, &zero, sizeof(unsigned int));
    }
    return e;
}

}  // namespace eup

