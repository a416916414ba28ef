// Partial-bounce-back forward step and its discrete adjoint.
//
// Forward model (Walsh, Burwinkle & Saar 2009, "A new partial-bounceback
// lattice-Boltzmann method for fluid flow through heterogeneous media"): with a
// solid fraction n_s(x) in [0,1] the post-collision state is
//   f*_i = (1 - n_s) BGK_i(f) + n_s f_opp(i),
// BGK_i the collision of CODE/SRC/col.F90 and f the streamed (pre-collision)
// populations.  n_s = 0 reproduces the plain step bit for bit.  The momentum
// the solid takes from node x is 2 n_s j(x), j = sum_i c_i f_i, so the drag of
// a step is F_x = sum_x 2 n_s j_x.
//
// Adjoint: the objective is J = sum_s gamma_s F_x(s) over the steps of the
// averaging window.  With lambda^s the adjoint of the state after step s and
// mu the adjoint of the streamed populations of step s,
//   mu_j     = (1-n_s) [J_BGK^T lambda^s]_j + n_s lambda^s_opp(j) + gamma_s 2 n_s c_jx
//   dJ/dn_s += sum_i lambda^s_i (f_opp(i) - BGK_i(f)) + gamma_s 2 j_x
//   lambda^{s-1}_j(x - c_j) = mu_j(x)                 (transpose of the pull)
// plus, for populations read through the halo, the transpose of the halo
// assignment that produced them (copies, outflow equilibria), which the host
// derives by running the reference's halo-block sequence on symbols.
#include <algorithm>
#include <string>
#include <vector>

#include "../../include/eup.h"
#include "internal.h"

namespace eup {

// ---------------------------------------------------------------------------
// Symbolic halo: what every halo slot holds after one step's halo blocks, as
// a function of the state entering the step.
// ---------------------------------------------------------------------------
namespace {

enum : int8_t { D_CONST = 0, D_COPY = 1, D_OUTFLOW = 2, D_STALE = 3 };
struct Desc {
    int8_t kind;
    int8_t q;     // source population (COPY) or produced population (OUTFLOW)
    int32_t idx;  // interior linear index (COPY) or (j-1) + (k-1)*m of x = l (OUTFLOW)
};

struct SymShell {
    const Geo& g;
    std::vector<Desc> d;
    std::vector<uint8_t> pass;
    int cur = 0;
    explicit SymShell(const Geo& g_) : g(g_), d((size_t)Q * g_.G, Desc{D_CONST, 0, 0}), pass((size_t)Q * g_.G, 0) {}
    size_t slot(int q, int i, int j, int k) const { return (size_t)q * g.G + (size_t)g.gidx(i, j, k); }
    Desc ld(int q1, int i, int j, int k) const {
        const int q = q1 - 1;
        if (g.interior(i, j, k)) return Desc{D_COPY, (int8_t)q, (int32_t)g.lin(i, j, k)};
        const size_t s = slot(q, i, j, k);
        Desc v = d[s];
        // written in the previous step and not yet in this one: a value of an older state
        if (cur == 2 && pass[s] == 1 && v.kind != D_CONST) v.kind = D_STALE;
        return v;
    }
    void st(int q1, int i, int j, int k, Desc v) {
        const size_t s = slot(q1 - 1, i, j, k);
        d[s] = v;
        pass[s] = (uint8_t)cur;
    }
};

// The halo blocks of CODE/SRC/bcond.bc.F90 in the reference's order, on
// symbols; the same ranges and assignments as the kernels of k_bc.cu.
void sym_halo_step(SymShell& S, const int bc[6]) {
    const Geo& g = S.g;
    const int l = g.l, m = g.m, n = g.n, l1 = l + 1, m1 = m + 1, n1 = n + 1;
    const Desc cst{D_CONST, 0, 0};
    auto LD = [&](int q, int i, int j, int k) { return S.ld(q, i, j, k); };
    auto ST = [&](int q, int i, int j, int k, Desc v) { S.st(q, i, j, k, v); };
    // front
    if (bc[0] == 0) {
        for (int k = 1; k <= n; ++k) {
            ST(12, l1, 0, k, LD(12, 1, m, k));
            for (int j = 1; j <= m; ++j)
                for (int q = 10; q <= 14; ++q) ST(q, l1, j, k, LD(q, 1, j, k));
        }
    } else if (bc[0] == 1) {
        for (int k = 1; k <= n; ++k)
            for (int j = 1; j <= m; ++j) {
                const Desc v1 = LD(1, l, j, k), v2 = LD(2, l, j, k), v3 = LD(3, l, j, k), v4 = LD(4, l, j, k),
                           v5 = LD(5, l, j, k);
                ST(12, l1, j - 1, k, v1);
                ST(13, l1, j, k - 1, v2);
                ST(10, l1, j + 1, k, v3);
                ST(11, l1, j, k + 1, v4);
                ST(14, l1, j, k, v5);
            }
    } else {
        for (int k = 1; k <= n; ++k)
            for (int j = 1; j <= m; ++j)
                for (int q = 10; q <= 14; ++q) ST(q, l1, j, k, Desc{D_OUTFLOW, (int8_t)(q - 1), (j - 1) + (k - 1) * m});
        for (int j = 1; j <= m; ++j)
            for (int q = 10; q <= 14; ++q) {
                const Desc lo = LD(q, l1, j, 1), hi = LD(q, l1, j, n);
                ST(q, l1, j, 0, lo);
                ST(q, l1, j, n1, hi);
            }
        for (int k = 1; k <= n; ++k)
            for (int q = 10; q <= 14; ++q) {
                const Desc lo = LD(q, l1, 1, k), hi = LD(q, l1, m, k);
                ST(q, l1, 0, k, lo);
                ST(q, l1, m1, k, hi);
            }
    }
    // rear
    if (bc[1] == 0) {
        for (int k = 1; k <= n; ++k) {
            ST(1, 0, m1, k, LD(1, l, 1, k));
            for (int j = 1; j <= m; ++j)
                for (int q = 1; q <= 5; ++q) ST(q, 0, j, k, LD(q, l, j, k));
        }
    } else if (bc[1] == 1) {
        for (int k = 1; k <= n; ++k)
            for (int j = 1; j <= m; ++j) {
                const Desc v10 = LD(10, 1, j, k), v11 = LD(11, 1, j, k), v12 = LD(12, 1, j, k),
                           v13 = LD(13, 1, j, k), v14 = LD(14, 1, j, k);
                ST(3, 0, j - 1, k, v10);
                ST(4, 0, j, k - 1, v11);
                ST(1, 0, j + 1, k, v12);
                ST(2, 0, j, k + 1, v13);
                ST(5, 0, j, k, v14);
            }
    } else {
        for (int k = 0; k <= n1; ++k)
            for (int j = 0; j <= m1; ++j)
                for (int q = 1; q <= 5; ++q) ST(q, 0, j, k, cst);
    }
    // up
    if (bc[4] == 0) {
        for (int j = 1; j <= m; ++j)
            for (int i = 1; i <= l; ++i) {
                const int qs[5] = {2, 9, 11, 15, 16};
                for (int q : qs) ST(q, i, j, n1, LD(q, i, j, 1));
            }
    } else if (bc[4] == 1 || bc[4] == 2) {
        for (int j = 1; j <= m; ++j)
            for (int i = 1; i <= l; ++i) {
                const Desc v6 = LD(6, i, j, n), v13 = LD(13, i, j, n), v18 = LD(18, i, j, n), v4 = LD(4, i, j, n),
                           v7 = LD(7, i, j, n);
                ST(15, i, j, n1, v6);
                ST(2, i - 1, j, n1, v13);
                ST(9, i, j - 1, n1, v18);
                ST(11, i + 1, j, n1, v4);
                ST(16, i, j + 1, n1, v7);
            }
    } else {
        for (int j = 0; j <= m1; ++j)
            for (int i = 0; i <= l1; ++i) {
                const Desc v6 = LD(6, i, j, n), v13 = LD(13, i, j, n), v18 = LD(18, i, j, n), v4 = LD(4, i, j, n),
                           v7 = LD(7, i, j, n);
                ST(15, i, j, n1, v6);
                ST(11, i, j, n1, v13);
                ST(16, i, j, n1, v18);
                ST(2, i, j, n1, v4);
                ST(9, i, j, n1, v7);
            }
    }
    // down
    for (int j = 1; j <= m; ++j)
        for (int i = 1; i <= l; ++i) {
            if (bc[5] == 0) {
                const int qs[5] = {4, 6, 7, 13, 18};
                for (int q : qs) ST(q, i, j, 0, LD(q, i, j, n));
            } else if (bc[5] == 1) {
                const Desc v15 = LD(15, i, j, 1), v11 = LD(11, i, j, 1), v16 = LD(16, i, j, 1), v2 = LD(2, i, j, 1),
                           v9 = LD(9, i, j, 1);
                ST(6, i, j, 0, v15);
                ST(4, i - 1, j, 0, v11);
                ST(7, i, j - 1, 0, v16);
                ST(13, i + 1, j, 0, v2);
                ST(18, i, j + 1, 0, v9);
            } else {
                const Desc v15 = LD(15, i, j, 1), v11 = LD(11, i, j, 1), v16 = LD(16, i, j, 1), v2 = LD(2, i, j, 1),
                           v9 = LD(9, i, j, 1);
                ST(6, i, j, 0, v15);
                ST(13, i, j, 0, v11);
                ST(18, i, j, 0, v16);
                ST(4, i, j, 0, v2);
                ST(7, i, j, 0, v9);
            }
        }
    // left
    for (int k = 1; k <= n; ++k) {
        if (bc[3] == 0) ST(3, 0, 0, k, LD(3, l, m, k));
        for (int i = 1; i <= l; ++i) {
            if (bc[3] == 0) {
                const int qs[5] = {3, 7, 8, 9, 12};
                Desc v[5];
                for (int t = 0; t < 5; ++t) v[t] = LD(qs[t], i, m, k);
                for (int t = 0; t < 5; ++t) ST(qs[t], i, 0, k, v[t]);
            } else if (bc[3] == 1) {
                const Desc v17 = LD(17, i, 1, k), v1 = LD(1, i, 1, k), v10 = LD(10, i, 1, k), v16 = LD(16, i, 1, k),
                           v18 = LD(18, i, 1, k);
                ST(8, i, 0, k, v17);
                ST(12, i + 1, 0, k, v1);
                ST(3, i - 1, 0, k, v10);
                ST(7, i, 0, k - 1, v16);
                ST(9, i, 0, k + 1, v18);
            } else {
                const Desc v17 = LD(17, i, 1, k), v1 = LD(1, i, 1, k), v10 = LD(10, i, 1, k), v16 = LD(16, i, 1, k),
                           v18 = LD(18, i, 1, k);
                ST(8, i, 0, k, v17);
                ST(3, i, 0, k, v1);
                ST(12, i, 0, k, v10);
                ST(9, i, 0, k, v16);
                ST(7, i, 0, k, v18);
            }
        }
    }
    // right
    for (int k = 1; k <= n; ++k) {
        if (bc[2] == 0) ST(10, l1, m1, k, LD(10, 1, 1, k));
        for (int i = 1; i <= l; ++i) {
            if (bc[2] == 0) {
                const int qs[5] = {1, 10, 16, 17, 18};
                Desc v[5];
                for (int t = 0; t < 5; ++t) v[t] = LD(qs[t], i, 1, k);
                for (int t = 0; t < 5; ++t) ST(qs[t], i, m1, k, v[t]);
            } else if (bc[2] == 1) {
                const Desc v3 = LD(3, i, m, k), v7 = LD(7, i, m, k), v8 = LD(8, i, m, k), v9 = LD(9, i, m, k),
                           v12 = LD(12, i, m, k);
                ST(10, i + 1, m1, k, v3);
                ST(16, i, m1, k + 1, v7);
                ST(17, i, m1, k, v8);
                ST(18, i, m1, k - 1, v9);
                ST(1, i - 1, m1, k, v12);
            } else {
                const Desc v3 = LD(3, i, m, k), v7 = LD(7, i, m, k), v8 = LD(8, i, m, k), v9 = LD(9, i, m, k),
                           v12 = LD(12, i, m, k);
                ST(1, i, m1, k, v3);
                ST(18, i, m1, k, v7);
                ST(17, i, m1, k, v8);
                ST(16, i, m1, k, v9);
                ST(10, i, m1, k, v12);
            }
        }
    }
    // free-slip edge fixes
    for (int i = 1; i <= l; ++i) {
        if (bc[3] == 3 && bc[4] == 3) ST(9, i, 0, n1, LD(18, i, 1, n));
        if (bc[2] == 3 && bc[4] == 3) ST(16, i, m1, n1, LD(7, i, m, n));
        if (bc[2] == 3 && bc[5] == 3) ST(18, i, m1, 0, LD(9, i, m, 1));
        if (bc[3] == 3 && bc[5] == 3) ST(7, i, 0, 0, LD(16, i, 1, 1));
    }
}

}  // namespace

int build_halo_adjoint_tables(const Geo& g, const int bc[6], HaloAdjointTables* out, std::string* err) {
    SymShell S(g);
    S.cur = 1;
    sym_halo_step(S, bc);
    S.cur = 2;
    sym_halo_step(S, bc);
    out->copy_key.clear();
    out->copy_start.clear();
    out->copy_slot.clear();
    out->out_jk.clear();
    out->out_start.clear();
    out->out_slot.clear();
    out->out_q.clear();
    struct CE { int64_t key; int64_t slot; };
    struct OE { int32_t jk; int64_t slot; int8_t q; };
    std::vector<CE> ce;
    std::vector<OE> oe;
    // pulled halo slots: (q, h) with h + c_q interior
    for (int q = 0; q < 18; ++q) {
        for (int k = 0; k <= g.n + 1; ++k)
            for (int j = 0; j <= g.m + 1; ++j)
                for (int i = 0; i <= g.l + 1; ++i) {
                    if (g.interior(i, j, k)) continue;
                    if (!g.interior(i + cx_of(q), j + cy_of(q), k + cz_of(q))) continue;
                    const size_t s = S.slot(q, i, j, k);
                    const Desc d = S.d[s];
                    if (d.kind == D_STALE) {
                        *err = "the adjoint needs every halo value of a step to follow from the state entering it; "
                               "with these boundary flags a halo block reads a value written one step earlier";
                        return EUP_ERR_UNSUPPORTED;
                    }
                    if (d.kind == D_COPY) ce.push_back(CE{(int64_t)d.q * g.N + d.idx, (int64_t)s});
                    if (d.kind == D_OUTFLOW) oe.push_back(OE{d.idx, (int64_t)s, d.q});
                }
    }
    std::sort(ce.begin(), ce.end(), [](const CE& a, const CE& b) { return a.key < b.key || (a.key == b.key && a.slot < b.slot); });
    for (size_t t = 0; t < ce.size(); ++t) {
        if (t == 0 || ce[t].key != ce[t - 1].key) {
            out->copy_key.push_back(ce[t].key);
            out->copy_start.push_back((int32_t)t);
        }
        out->copy_slot.push_back(ce[t].slot);
    }
    out->copy_start.push_back((int32_t)ce.size());
    std::sort(oe.begin(), oe.end(), [](const OE& a, const OE& b) {
        return a.jk < b.jk || (a.jk == b.jk && (a.q < b.q || (a.q == b.q && a.slot < b.slot)));
    });
    for (size_t t = 0; t < oe.size(); ++t) {
        if (t == 0 || oe[t].jk != oe[t - 1].jk) {
            out->out_jk.push_back(oe[t].jk);
            out->out_start.push_back((int32_t)t);
        }
        out->out_slot.push_back(oe[t].slot);
        out->out_q.push_back(oe[t].q);
    }
    out->out_start.push_back((int32_t)oe.size());
    return EUP_OK;
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
namespace {

// Values of a state stored as S, worked on in R: the populations f themselves (FP32/FP64
// storage), or for 16-bit storage the scaled deviations D = (f - w) S in the step kernels
// ("kernel values", as the stream-collide kernels use them) and f in the adjoint.
template <typename S, typename R>
struct PState {
    static constexpr bool dev = DevStore<S>::value;
    static __device__ __forceinline__ R kval(S raw) {
        if constexpr (dev) return DevStore<S>::to_f(raw);
        else return raw;
    }
    static __device__ __forceinline__ S kstore(R v) {
        if constexpr (dev) return DevStore<S>::from_f(v);
        else return v;
    }
    // kernel value of population q pulled to node (i, j, k) (linear index lin)
    static __device__ __forceinline__ R pull_k(const Lat<S, R>& L, const Geo& g, int q, int i, int j, int k,
                                               int64_t lin, bool face) {
        if (!face) return kval(L.pop[q][lin - cx_of(q) - (int64_t)cy_of(q) * g.l - (int64_t)cz_of(q) * g.lm]);
        const int si = i - cx_of(q), sj = j - cy_of(q), sk = k - cz_of(q);
        if (g.interior(si, sj, sk)) return kval(L.pop[q][g.lin(si, sj, sk)]);
        const R f = L.ghost[(int64_t)q * g.G + g.gidx(si, sj, sk)];
        if constexpr (dev) return (f - weight<R>(q)) * L.scale;
        else return f;
    }
    // population f_q pulled to node (i, j, k)
    static __device__ __forceinline__ R pull_f(const Lat<S, R>& L, const Geo& g, int q, int i, int j, int k,
                                               int64_t lin, bool face) {
        if (!face)
            return Store<S, R>::load(L.pop[q][lin - cx_of(q) - (int64_t)cy_of(q) * g.l - (int64_t)cz_of(q) * g.lm], q,
                                     L.inv_scale);
        return lat_load(L, g, q, i - cx_of(q), j - cy_of(q), k - cz_of(q));
    }
    static __device__ __forceinline__ R f_of(const Lat<S, R>& L, int q, int64_t lin) {
        return Store<S, R>::load(L.pop[q][lin], q, L.inv_scale);
    }
};

template <typename R>
__device__ __forceinline__ R pull_pre(const Lat<R, R>& L, const Geo& g, int q, int i, int j, int k, int64_t lin,
                                      bool face) {
    return PState<R, R>::pull_f(L, g, q, i, j, k, lin, face);
}

// The partial-bounce-back step is the plain stream-collide (every node's BGK value, the
// same kernels and bits as the plain step) followed by this kernel over the list of
// voxels with n_s > 0: it pulls their pre-collision populations again, mixes
//   f*_q = (1 - n_s) BGK_q + n_s f_opp(q)
// into the destination lattice (and its x-face copy), and with `series` adds the
// momentum the solid takes, F = sum 2 n_s j(x) over the list, j the momentum of the pulled
// populations, in FP64 into series[(itime + 1) % cap], advancing the device step counter
// (one block at least, so an empty list records a zero force).
template <typename S, typename R>
__global__ void __launch_bounds__(256) k_pbb_list(Lat<S, R> src, Lat<S, R> dst, Geo g, const R* ns,
                                                  const int32_t* list, int64_t nlist, Reduce red, double* series,
                                                  int64_t cap, int64_t* d_itime) {
    using P = PState<S, R>;
    double f[3] = {0.0, 0.0, 0.0};
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nlist;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int32_t l32 = list[t];  // one lattice holds fewer than 2^31 nodes
        const int64_t lin = l32;
        const int row = l32 / g.l;
        const int i = l32 - row * g.l + 1, j = row % g.m + 1, k = row / g.m + 1;
        const bool face = (i == 1) | (i == g.l) | (j == 1) | (j == g.m) | (k == 1) | (k == g.n);
        // every load before the first store (the stores go to the lattice the BGK values are
        // read from, so loads after them could not be issued ahead); kernel values: f, or the
        // deviations D for 16-bit storage, where the mixing is the same (w_q = w_opp(q))
        R pre[19], x[19];
#pragma unroll
        for (int q = 0; q < 18; ++q) pre[q] = P::pull_k(src, g, q, i, j, k, lin, face);
        pre[18] = P::kval(src.pop[18][lin]);
#pragma unroll
        for (int q = 0; q < 19; ++q) x[q] = P::kval(dst.pop[q][lin]);
        const R s = ns[lin], s1 = R(1) - s;
        if (series) {
            double jx = 0.0, jy = 0.0, jz = 0.0;
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                jx += (q == 18 ? 0 : cx_of(q)) * (double)pre[q];
                jy += (q == 18 ? 0 : cy_of(q)) * (double)pre[q];
                jz += (q == 18 ? 0 : cz_of(q)) * (double)pre[q];
            }
            // sum_q c_q w_q = 0: the momentum of the deviations is the momentum
            const double js = P::dev ? 1.0 / (double)src.scale : 1.0;
            f[0] += 2.0 * (double)s * (jx * js);
            f[1] += 2.0 * (double)s * (jy * js);
            f[2] += 2.0 * (double)s * (jz * js);
        }
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const S v = P::kstore(s1 * x[q] + s * pre[opp_of(q)]);
            dst.pop[q][lin] = v;
            if (q < 18 && (i == 1 || i == g.l)) {
                const R fv = Store<S, R>::load(v, q, dst.inv_scale);  // what a later load returns
                if (i == 1) dst.xface[xface_idx(g, 0, q, j, k)] = fv;
                if (i == g.l) dst.xface[xface_idx(g, 1, q, j, k)] = fv;
            }
        }
    }
    if (series) block_reduce_store<3>(f, red, nullptr, series, cap, d_itime, 1, 1);
}

// c_q . (x, y, z) with the zero components of c_q left out at compile time (q a constant
// once the loops over q are unrolled): a product by a zero component is not folded away
// under IEEE rules, and most of these products are by zero.
template <typename R>
__device__ __forceinline__ R cdot(int q, R x, R y, R z) {
    const int c[3] = {q == 18 ? 0 : cx_of(q), q == 18 ? 0 : cy_of(q), q == 18 ? 0 : cz_of(q)};
    const R v[3] = {x, y, z};
    R acc = R(0);
    bool any = false;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (c[d] == 0) continue;
        const R term = c[d] > 0 ? v[d] : -v[d];
        acc = any ? acc + term : term;
        any = true;
    }
    return acc;
}

// Adjoint of one step: state f (entering the step, its halo shell holding the
// halo values of that step), lam_in = adjoint of the state the step produced;
// writes the adjoint of f (lam_out, pushed), the halo part of it (gmu, per
// halo slot), and accumulates dJ/dn_s.  Everything the transpose of the BGK
// Jacobian needs from lam comes from ten weighted moments of it (sum w lam,
// sum w lam c_a, sum w lam c_a c_b) and sum lam c_x, and dJ/dn_s from sum lam f,
// sum lam f_opp and the same moments (sum lam f_eq is quadratic in u), so each
// direction costs a few signed additions instead of an equilibrium evaluation.
// FACE: the node lies on one of the six boundary planes (its pulls and pushes may cross the
// halo); the interior kernel is compiled without that code.
template <typename S, typename R, bool FACE>
__device__ __forceinline__ void adjoint_node(const Lat<S, R>& f, const Geo& g, const Phys<R>& ph, const R* ns,
                                             const Lat<R, R>& lam_in, const Lat<R, R>& lam_out, R* gmu,
                                             double* grad, R gamma, int i, int j, int k) {
    {
        const int64_t lin = (int64_t)(i - 1) + (int64_t)g.l * ((j - 1) + (int64_t)g.m * (k - 1));
        constexpr bool face = FACE;
        R pre[19], lam[19];
#pragma unroll
        for (int q = 0; q < 18; ++q) pre[q] = PState<S, R>::pull_f(f, g, q, i, j, k, lin, face);
        pre[18] = PState<S, R>::f_of(f, 18, lin);
#pragma unroll
        for (int q = 0; q < 19; ++q) lam[q] = lam_in.pop[q][lin];
        const R s = ns[lin], s1 = R(1) - s;
        R rho = pre[0], jx = pre[0], jy = -pre[0], jz = R(0);
        R lp = lam[0] * pre[0], lpo = lam[0] * pre[opp_of(0)];  // sum lam_q f_q, sum lam_q f_opp(q)
#pragma unroll
        for (int q = 1; q < 19; ++q) {
            rho += pre[q];
            const int cx = q == 18 ? 0 : cx_of(q), cy = q == 18 ? 0 : cy_of(q), cz = q == 18 ? 0 : cz_of(q);
            if (cx != 0) jx = cx > 0 ? jx + pre[q] : jx - pre[q];
            if (cy != 0) jy = cy > 0 ? jy + pre[q] : jy - pre[q];
            if (cz != 0) jz = cz > 0 ? jz + pre[q] : jz - pre[q];
            lp += lam[q] * pre[q];
            lpo += lam[q] * pre[opp_of(q)];
        }
        const R ux = jx / rho, uy = jy / rho, uz = jz / rho;
        const R usq = ux * ux + uy * uy + uz * uz;
        // moments of lam: sum lam c_a c_b (ab = xx, yy, zz, xy, xz, yz), sum lam c_a and sum lam
        // over the axis (w = 1/18) and diagonal (w = 1/36) directions apart; c has components 0
        // and +-1, so each is a signed sum
        R m0[2] = {R(0), R(0)}, m1[2][3] = {}, m2[2][6] = {};
#pragma unroll
        for (int q = 0; q < 18; ++q) {
            const int cls = wclass_of(q) == 1 ? 0 : 1;
            const int c[3] = {cx_of(q), cy_of(q), cz_of(q)};
            const R v = lam[q];
            m0[cls] += v;
#pragma unroll
            for (int d = 0; d < 3; ++d)
                if (c[d] != 0) m1[cls][d] = c[d] > 0 ? m1[cls][d] + v : m1[cls][d] - v;
#pragma unroll
            for (int d = 0; d < 3; ++d)
                if (c[d] != 0) m2[cls][d] += v;  // c_d^2 = 1
            const int pr[3][2] = {{0, 1}, {0, 2}, {1, 2}};
#pragma unroll
            for (int e = 0; e < 3; ++e) {
                const int cc = c[pr[e][0]] * c[pr[e][1]];
                if (cc != 0) m2[cls][3 + e] = cc > 0 ? m2[cls][3 + e] + v : m2[cls][3 + e] - v;
            }
        }
        const R p0 = weight<R>(18), p1 = weight<R>(4), p2 = weight<R>(0);
        const R L0 = p0 * lam[18] + p1 * m0[0] + p2 * m0[1];           // sum w lam
        R L1[3], L2[6];
#pragma unroll
        for (int d = 0; d < 3; ++d) L1[d] = p1 * m1[0][d] + p2 * m1[1][d];  // sum w lam c
#pragma unroll
        for (int e = 0; e < 6; ++e) L2[e] = p1 * m2[0][e] + p2 * m2[1][e];  // sum w lam c c
        const R fxu = m1[0][0] + m1[1][0];                                  // sum lam c_x
        const R uL1 = ux * L1[0] + uy * L1[1] + uz * L1[2];
        const R L2u[3] = {L2[0] * ux + L2[3] * uy + L2[4] * uz, L2[3] * ux + L2[1] * uy + L2[5] * uz,
                          L2[4] * ux + L2[5] * uy + L2[2] * uz};
        const R uL2u = ux * L2u[0] + uy * L2u[1] + uz * L2u[2];
        const R c15 = R(1.5) * usq;
        // sum lam f_eq = rho (L0 (1 - 1.5 u^2) + 3 u.L1 + 4.5 u.L2.u); the step's BGK value is
        // omega1 f + omega f_eq + fgrad rho c_x
        const R lfeq = rho * (L0 * (R(1) - c15) + R(3) * uL1 + R(4.5) * uL2u);
        const R lbgk = ph.omega1 * lp + ph.omega * lfeq + ph.fgrad * rho * fxu;
        const R gs = R(2) * gamma * jx + (lpo - lbgk);  // dJ/dn_s of this step
        // transpose of the BGK Jacobian through rho and u:
        //   A = s1 sum w lam (1 - 4.5 (c.u)^2 + 1.5 u^2), B = s1 (3 (L1 - u L0) + 9 L2 u), Fx = s1 sum lam c_x
        const R A = s1 * (L0 * (R(1) + c15) - R(4.5) * uL2u);
        const R Bx = s1 * (R(3) * (L1[0] - ux * L0) + R(9) * L2u[0]);
        const R By = s1 * (R(3) * (L1[1] - uy * L0) + R(9) * L2u[1]);
        const R Bz = s1 * (R(3) * (L1[2] - uz * L0) + R(9) * L2u[2]);
        const R Fx = s1 * fxu;
        grad[lin] += (double)gs;
        const R common = ph.omega * A + ph.fgrad * Fx;
        const R g2 = gamma * R(2) * s;
        const R o1s1 = ph.omega1 * s1;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const int cx = q == 18 ? 0 : cx_of(q), cy = q == 18 ? 0 : cy_of(q), cz = q == 18 ? 0 : cz_of(q);
            R mu = o1s1 * lam[q] + common;
            if (cx != 0 || cy != 0 || cz != 0) mu = mu + ph.omega * cdot<R>(q, Bx, By, Bz);
            mu = mu + s * lam[opp_of(q)];
            if (cx != 0) mu = cx > 0 ? mu + g2 : mu - g2;
            if (!face) {  // f_q(x) was pulled from the interior node x - c_q
                lam_out.pop[q][lin - cx - (int64_t)cy * g.l - (int64_t)cz * g.lm] = mu;
            } else {
                const int si = i - cx, sj = j - cy, sk = k - cz;
                if (g.interior(si, sj, sk)) lam_out.pop[q][g.lin(si, sj, sk)] = mu;
                else gmu[(int64_t)q * g.G + g.gidx(si, sj, sk)] = mu;
                // no interior node pulls f_q(x) when x + c_q is outside: start that slot at zero
                if (!g.interior(i + cx, j + cy, k + cz)) lam_out.pop[q][lin] = R(0);
            }
        }
    }
}

// Nodes with 2 <= i <= l-1, 2 <= j <= m-1, 2 <= k <= n-1, one per thread; grid
// (ceil((l-2)/128), m-2, n-2): indices from the block coordinates, no halo code.
template <typename S, typename R, int MINB>
__global__ void __launch_bounds__(128, MINB) k_pbb_adjoint(Lat<S, R> f, Geo g, Phys<R> ph, const R* ns,
                                                           Lat<R, R> lam_in, Lat<R, R> lam_out, R* gmu,
                                                           double* grad, R gamma) {
    const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x) + 2;
    if (i > g.l - 1) return;
    adjoint_node<S, R, false>(f, g, ph, ns, lam_in, lam_out, gmu, grad, gamma, i, (int)blockIdx.y + 2,
                           (int)blockIdx.z + 2);
}

// The rest: every node of the rows on the y/z boundary planes (face rows f < nfr, in the
// order of face_row), then the columns i = 1 and i = l of the other rows.
template <typename S, typename R>
__global__ void __launch_bounds__(128) k_pbb_adjoint_faces(Lat<S, R> f, Geo g, Phys<R> ph, const R* ns,
                                                           Lat<R, R> lam_in, Lat<R, R> lam_out, R* gmu,
                                                           double* grad, R gamma, int nfr, int64_t nitems) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nitems) return;
    int i, j, k;
    if (t < (int64_t)nfr * g.l) {
        const int fr = (int)(t / g.l);
        i = (int)(t - (int64_t)fr * g.l) + 1;
        face_row(g, fr, &j, &k);
    } else {
        const int sides = g.l == 1 ? 1 : 2;
        const int u = (int)(t - (int64_t)nfr * g.l);
        const int r = u / sides, side = u - r * sides;
        j = r % (g.m - 2) + 2;
        k = r / (g.m - 2) + 2;
        i = side ? g.l : 1;
    }
    adjoint_node<S, R, true>(f, g, ph, ns, lam_in, lam_out, gmu, grad, gamma, i, j, k);
}

// Halo values copied from interior populations: add their adjoints back, one
// thread per source, sources' halo slots summed in a fixed order.
template <typename R>
__global__ void k_adj_copy(Geo g, const int64_t* key, const int32_t* start, const int64_t* slot, int64_t nkey,
                           const R* gmu, Lat<R, R> lam_out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nkey) return;
    R acc = R(0);
    for (int32_t e = start[t]; e < start[t + 1]; ++e) acc += gmu[slot[e]];
    const int q = (int)(key[t] / g.N);
    const int64_t lin = key[t] % g.N;
    lam_out.pop[q][lin] += acc;
}

// Outflow halo values (equilibria of the momentum of x = l,
// CODE/SRC/bcond.bc.F90:138-165): propagate their adjoints to the 18 moving
// populations of the node they were computed from.
template <typename S, typename R>
__global__ void k_adj_outflow(Geo g, const int32_t* jk, const int32_t* start, const int64_t* slot, const int8_t* qo,
                              int64_t nsrc, const R* gmu, Lat<S, R> f, Lat<R, R> lam_out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nsrc) return;
    const int j = jk[t] % g.m + 1, k = jk[t] / g.m + 1;
    const int64_t lin = g.lin(g.l, j, k);
    R J[3] = {R(0), R(0), R(0)};
    R a[18];
#pragma unroll
    for (int q = 0; q < 18; ++q) a[q] = PState<S, R>::f_of(f, q, lin);
    J[0] = a[0] + a[1] + a[2] + a[3] + a[4] - a[9] - a[10] - a[11] - a[12] - a[13];
    J[1] = a[2] + a[6] + a[7] + a[8] + a[11] - a[0] - a[9] - a[15] - a[16] - a[17];
    J[2] = a[3] + a[5] + a[6] + a[12] + a[17] - a[1] - a[8] - a[10] - a[14] - a[15];
    R psi[3] = {R(0), R(0), R(0)};
    for (int32_t e = start[t]; e < start[t + 1]; ++e) {
        const int q = qo[e];
        const R mu = gmu[slot[e]];
        const R c[3] = {R(cx_of(q)), R(cy_of(q)), R(cz_of(q))};
        const R cJ = c[0] * J[0] + c[1] * J[1] + c[2] * J[2];
        const R w = weight<R>(q);
        for (int a3 = 0; a3 < 3; ++a3) psi[a3] += mu * w * (R(3) * c[a3] + R(1.5) * (R(6) * cJ * c[a3] - R(2) * J[a3]));
    }
    // all 18 values of the node first, then the updated ones (a load after a store through
    // another population's pointer would wait for it)
    R old[18];
#pragma unroll
    for (int p = 0; p < 18; ++p) old[p] = lam_out.pop[p][lin];
#pragma unroll
    for (int p = 0; p < 18; ++p)
        lam_out.pop[p][lin] = old[p] + (R(cx_of(p)) * psi[0] + R(cy_of(p)) * psi[1] + R(cz_of(p)) * psi[2]);
}

unsigned capped_grid(int64_t work, int tpb) {
    int64_t b = (work + tpb - 1) / tpb;
    if (b < 1) b = 1;
    if (b > kReduceMaxBlocks) b = kReduceMaxBlocks;
    return (unsigned)b;
}

}  // namespace

template <typename S, typename R>
void launch_pbb_step(const Lat<S, R>& src, const Lat<S, R>& dst, const Geo& g, const Phys<R>& ph, const R* ns,
                     const int32_t* ns_list, int64_t ns_count, const Reduce& red, double* series, int64_t cap,
                     int64_t* d_itime, cudaStream_t st) {
    launch_stream_collide<S, R>(src, dst, g, ph, 0, st);
    k_pbb_list<S, R><<<capped_grid(ns_count, 256), 256, 0, st>>>(src, dst, g, ns, ns_list, ns_count, red, series,
                                                                  cap, d_itime);
}

template <typename S, typename R>
void launch_pbb_adjoint(const Lat<S, R>& f, const Geo& g, const Phys<R>& ph, const R* ns, const Lat<R, R>& lam_in,
                        const Lat<R, R>& lam_out, R* gmu, double* grad, R gamma, const HaloAdjointDevice& t,
                        cudaStream_t st, int parts) {
    // resident blocks of 128 per SM the registers are sized for: FP32 arithmetic 6 (80
    // registers), FP64 4
    if ((parts & kAdjInterior) && g.l > 2 && g.m > 2 && g.n > 2) {
        const dim3 grid((unsigned)((g.l - 2 + 127) / 128), (unsigned)(g.m - 2), (unsigned)(g.n - 2));
        k_pbb_adjoint<S, R, sizeof(R) == 4 ? 6 : 4><<<grid, 128, 0, st>>>(f, g, ph, ns, lam_in, lam_out, gmu, grad,
                                                                           gamma);
    }
    if (parts & kAdjFaces) {
        const int nz = g.n >= 2 ? 2 : 1, ny = g.m >= 2 ? 2 : 1;
        const int nfr = nz * g.m + (g.n > 2 ? (g.n - 2) * ny : 0);
        const int64_t inner_rows = (g.m > 2 && g.n > 2) ? (int64_t)(g.m - 2) * (g.n - 2) : 0;
        const int64_t nitems = (int64_t)nfr * g.l + inner_rows * (g.l == 1 ? 1 : 2);
        k_pbb_adjoint_faces<S, R><<<(unsigned)((nitems + 127) / 128), 128, 0, st>>>(f, g, ph, ns, lam_in, lam_out,
                                                                                     gmu, grad, gamma, nfr, nitems);
    }
    if (!(parts & kAdjTransposes)) return;
    if (t.ncopy > 0)
        // small blocks: a few thousand threads still spread over every SM
        k_adj_copy<R><<<(unsigned)((t.ncopy + 63) / 64), 64, 0, st>>>(g, t.copy_key, t.copy_start, t.copy_slot,
                                                                       t.ncopy, gmu, lam_out);
    if (t.nout > 0)
        k_adj_outflow<S, R><<<(unsigned)((t.nout + 63) / 64), 64, 0, st>>>(g, t.out_jk, t.out_start, t.out_slot,
                                                                            t.out_q, t.nout, gmu, f, lam_out);
}

#define EUP_PBB_INST(S, R)                                                                                       \
    template void launch_pbb_step<S, R>(const Lat<S, R>&, const Lat<S, R>&, const Geo&, const Phys<R>&, const R*, \
                                        const int32_t*, int64_t, const Reduce&, double*, int64_t, int64_t*,        \
                                        cudaStream_t);                                                             \
    template void launch_pbb_adjoint<S, R>(const Lat<S, R>&, const Geo&, const Phys<R>&, const R*,                \
                                           const Lat<R, R>&, const Lat<R, R>&, R*, double*, R,                     \
                                           const HaloAdjointDevice&, cudaStream_t, int);
EUP_PBB_INST(float, float)
EUP_PBB_INST(double, double)
EUP_PBB_INST(__half, float)
EUP_PBB_INST(__nv_bfloat16, float)

}  // namespace eup
