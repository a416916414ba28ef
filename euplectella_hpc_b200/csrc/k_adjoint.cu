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

template <typename R>
__device__ __forceinline__ R pull_pre(const Lat<R, R>& L, const Geo& g, int q, int i, int j, int k, int64_t lin,
                                      bool face) {
    if (!face) return L.pop[q][lin - cx_of(q) - (int64_t)cy_of(q) * g.l - (int64_t)cz_of(q) * g.lm];
    return lat_load(L, g, q, i - cx_of(q), j - cy_of(q), k - cz_of(q));
}

// Forward partial-bounce-back step, one node per thread (FP64 storage, odd l).  The force
// of the step is k_pbb_force's.
template <typename R>
__global__ void __launch_bounds__(256) k_pbb_step(Lat<R, R> src, Lat<R, R> dst, Geo g, Phys<R> ph, const R* ns) {
    for (int64_t lin = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; lin < g.N;
         lin += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(lin % g.l) + 1, j = (int)((lin / g.l) % g.m) + 1, k = (int)(lin / g.lm) + 1;
        const bool face = (i == 1) | (i == g.l) | (j == 1) | (j == g.m) | (k == 1) | (k == g.n);
        R x[19];
#pragma unroll
        for (int q = 0; q < 18; ++q) x[q] = pull_pre(src, g, q, i, j, k, lin, face);
        x[18] = src.pop[18][lin];
        collide<R>(x, ph.omega, ph.omega1, ph.fgrad);
        const R s = ns[lin];
        if (s != R(0)) {  // f* = (1 - n_s) BGK(f) + n_s f_opp; n_s = 0 leaves the BGK value
            const R s1 = R(1) - s;
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                const int qo = opp_of(q);
                const R pre_o = qo == 18 ? src.pop[18][lin] : pull_pre(src, g, qo, i, j, k, lin, face);
                x[q] = s1 * x[q] + s * pre_o;
            }
        }
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            dst.pop[q][lin] = x[q];
            if (q < 18 && i == 1) dst.xface[xface_idx(g, 0, q, j, k)] = x[q];
            if (q < 18 && i == g.l) dst.xface[xface_idx(g, 1, q, j, k)] = x[q];
        }
    }
}

// Pulled population q of the pair (i, i+1), i odd, of row (j, k) (rowlin = linear index of
// x = 1 on the row): rows on the y/z boundary planes node by node through the halo shell,
// elsewhere two shifted loads (one 8-byte load when cx = 0) with the x-halo values of the
// row's first and last node from the shell.
__device__ __forceinline__ F2 pull_pair_f32(const Lat<float, float>& L, const Geo& g, int q, int i, int j, int k,
                                            int rowlin, bool face) {
    const int cx = q == 18 ? 0 : cx_of(q), cy = q == 18 ? 0 : cy_of(q), cz = q == 18 ? 0 : cz_of(q);
    if (face) return F2(lat_load(L, g, q, i - cx, j - cy, k - cz), lat_load(L, g, q, i + 1 - cx, j - cy, k - cz));
    const float* rp = L.pop[q] + (rowlin - cy * g.l - cz * (int)g.lm);
    if (cx == 0) return F2(*reinterpret_cast<const float2*>(rp + (i - 1)));
    // both loads stay inside the population for interior rows (see the stream-collide kernel)
    float a = rp[i - 1 - cx], b = rp[i - cx];
    if (cx == 1 && i == 1) a = L.ghost[(int64_t)q * g.G + g.gidx(0, j - cy, k - cz)];
    if (cx == -1 && i + 1 == g.l) b = L.ghost[(int64_t)q * g.G + g.gidx(g.l + 1, j - cy, k - cz)];
    return F2(a, b);
}

// Forward partial-bounce-back step, FP32, two nodes per thread (l even): the BGK collision
// runs once on F2 values (packed FP32, each lane rounded as the one-node kernel, so the
// bits are the same), and only pairs with n_s != 0 on either node pull the opposite
// populations again for the mixing.  grid (ceil(np/128), m, n), pairs p0 .. p0+np-1.
template <int MINB>
__global__ void __launch_bounds__(128, MINB) k_pbb_pair(Lat<float, float> src, Lat<float, float> dst, Geo g,
                                                        Phys<float> ph, const float* ns, int np) {
    const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (t >= np) return;
    const int i = 2 * t + 1, j = (int)blockIdx.y + 1, k = (int)blockIdx.z + 1;
    const int rowlin = g.l * ((j - 1) + g.m * (k - 1));
    const bool face = (j == 1) | (j == g.m) | (k == 1) | (k == g.n);
    F2 x[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) x[q] = pull_pair_f32(src, g, q, i, j, k, rowlin, face);
    collide<F2>(x, F2(ph.omega), F2(ph.omega1), F2(ph.fgrad));
    const float2 sv = *reinterpret_cast<const float2*>(ns + rowlin + (i - 1));
    if (sv.x != 0.0f || sv.y != 0.0f) {
        const F2 s(sv), s1 = F2(1.0f) - s;
#pragma unroll
        for (int q = 0; q < 19; ++q) x[q] = s1 * x[q] + s * pull_pair_f32(src, g, opp_of(q), i, j, k, rowlin, face);
    }
    if (i == 1) {
#pragma unroll
        for (int q = 0; q < 18; ++q) dst.xface[xface_idx(g, 0, q, j, k)] = x[q].v.x;
    }
    if (i + 1 == g.l) {
#pragma unroll
        for (int q = 0; q < 18; ++q) dst.xface[xface_idx(g, 1, q, j, k)] = x[q].v.y;
    }
#pragma unroll
    for (int q = 0; q < 19; ++q) *reinterpret_cast<float2*>(dst.pop[q] + rowlin + (i - 1)) = x[q].v;
}

// Momentum the solid takes in the step, F = sum over voxels with n_s > 0 of 2 n_s j(x), j
// the momentum of the pulled (pre-collision) populations, in FP64 over the list of those
// voxels; written to series[(itime + 1) % cap] and the device step counter advanced (one
// block at least, so an empty list records a zero force).
template <typename R>
__global__ void __launch_bounds__(256) k_pbb_force(Lat<R, R> src, Geo g, const R* ns, const int32_t* list,
                                                   int64_t nlist, Reduce red, double* series, int64_t cap,
                                                   int64_t* d_itime) {
    double f[3] = {0.0, 0.0, 0.0};
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nlist;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t lin = list[t];
        const int i = (int)(lin % g.l) + 1, j = (int)((lin / g.l) % g.m) + 1, k = (int)(lin / g.lm) + 1;
        const bool face = (i == 1) | (i == g.l) | (j == 1) | (j == g.m) | (k == 1) | (k == g.n);
        double jx = 0.0, jy = 0.0, jz = 0.0;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const double v = (double)(q == 18 ? src.pop[18][lin] : pull_pre(src, g, q, i, j, k, lin, face));
            jx += (q == 18 ? 0 : cx_of(q)) * v;
            jy += (q == 18 ? 0 : cy_of(q)) * v;
            jz += (q == 18 ? 0 : cz_of(q)) * v;
        }
        const double s = (double)ns[lin];
        f[0] += 2.0 * s * jx;
        f[1] += 2.0 * s * jy;
        f[2] += 2.0 * s * jz;
    }
    block_reduce_store<3>(f, red, nullptr, series, cap, d_itime, 1, 1);
}

// Adjoint of one step: state f (entering the step, its halo shell holding the
// halo values of that step), lam_in = adjoint of the state the step produced;
// writes the adjoint of f (lam_out, pushed), the halo part of it (gmu, per
// halo slot), and accumulates dJ/dn_s.  The pulled populations stay in registers;
// lam_in is read in two passes over the 19 directions (the sums of the BGK
// Jacobian's transpose first, then the pushed values, whose second read of the
// node's 19 words comes from the cache), so one node fits in few registers and
// many nodes are in flight per SM.  The BGK post-collision value needed by dJ/dn_s
// is re-evaluated from rho and u.
template <typename R, int MINB>
__global__ void __launch_bounds__(256, MINB) k_pbb_adjoint(Lat<R, R> f, Geo g, Phys<R> ph, const R* ns, Lat<R, R> lam_in,
                                                     Lat<R, R> lam_out, R* gmu, double* grad, R gamma) {
    for (int64_t lin = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; lin < g.N;
         lin += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(lin % g.l) + 1, j = (int)((lin / g.l) % g.m) + 1, k = (int)(lin / g.lm) + 1;
        const bool face = (i == 1) | (i == g.l) | (j == 1) | (j == g.m) | (k == 1) | (k == g.n);
        R pre[19];
#pragma unroll
        for (int q = 0; q < 18; ++q) pre[q] = pull_pre(f, g, q, i, j, k, lin, face);
        pre[18] = f.pop[18][lin];
        const R s = ns[lin], s1 = R(1) - s;
        R rho = R(0), jx = R(0), jy = R(0), jz = R(0);
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            rho += pre[q];
            jx += R(cx_of(q)) * pre[q];
            jy += R(cy_of(q)) * pre[q];
            jz += R(cz_of(q)) * pre[q];
        }
        const R ux = jx / rho, uy = jy / rho, uz = jz / rho;
        const R usq = ux * ux + uy * uy + uz * uz;
        const R frho = ph.fgrad * rho;
        R gs = R(2) * gamma * jx;  // dJ/dn_s of this step
        R A = R(0), Bx = R(0), By = R(0), Bz = R(0), Fx = R(0);
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const R lam = lam_in.pop[q][lin];
            const R w = weight<R>(q);
            const R cu = R(cx_of(q)) * ux + R(cy_of(q)) * uy + R(cz_of(q)) * uz;
            const R feq = w * rho * (R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * usq);
            const R bgk = ph.omega1 * pre[q] + ph.omega * feq + frho * R(cx_of(q));
            gs += lam * (pre[opp_of(q)] - bgk);
            const R nw = s1 * lam * w;
            A += nw * (R(1) - R(4.5) * cu * cu + R(1.5) * usq);
            const R b9 = nw * R(9) * cu;
            Bx += nw * R(3) * (R(cx_of(q)) - ux) + b9 * R(cx_of(q));
            By += nw * R(3) * (R(cy_of(q)) - uy) + b9 * R(cy_of(q));
            Bz += nw * R(3) * (R(cz_of(q)) - uz) + b9 * R(cz_of(q));
            Fx += s1 * lam * R(cx_of(q));
        }
        grad[lin] += (double)gs;
        const R common = ph.omega * A + ph.fgrad * Fx;
        const R g2 = gamma * R(2) * s;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const R lam = lam_in.pop[q][lin], lam_o = lam_in.pop[opp_of(q)][lin];
            const R mu = ph.omega1 * s1 * lam + common +
                         ph.omega * (R(cx_of(q)) * Bx + R(cy_of(q)) * By + R(cz_of(q)) * Bz) +
                         s * lam_o + g2 * R(cx_of(q));
            if (!face) {  // f_q(x) was pulled from the interior node x - c_q
                lam_out.pop[q][lin - cx_of(q) - (int64_t)cy_of(q) * g.l - (int64_t)cz_of(q) * g.lm] = mu;
            } else {
                const int si = i - cx_of(q), sj = j - cy_of(q), sk = k - cz_of(q);
                if (g.interior(si, sj, sk)) lam_out.pop[q][g.lin(si, sj, sk)] = mu;
                else gmu[(int64_t)q * g.G + g.gidx(si, sj, sk)] = mu;
                // no interior node pulls f_q(x) when x + c_q is outside: start that slot at zero
                if (!g.interior(i + cx_of(q), j + cy_of(q), k + cz_of(q))) lam_out.pop[q][lin] = R(0);
            }
        }
    }
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
template <typename R>
__global__ void k_adj_outflow(Geo g, const int32_t* jk, const int32_t* start, const int64_t* slot, const int8_t* qo,
                              int64_t nsrc, const R* gmu, Lat<R, R> f, Lat<R, R> lam_out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nsrc) return;
    const int j = jk[t] % g.m + 1, k = jk[t] / g.m + 1;
    const int64_t lin = g.lin(g.l, j, k);
    R J[3] = {R(0), R(0), R(0)};
    R a[18];
#pragma unroll
    for (int q = 0; q < 18; ++q) a[q] = f.pop[q][lin];
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
#pragma unroll
    for (int p = 0; p < 18; ++p)
        lam_out.pop[p][lin] += R(cx_of(p)) * psi[0] + R(cy_of(p)) * psi[1] + R(cz_of(p)) * psi[2];
}

unsigned capped_grid(int64_t work, int tpb) {
    int64_t b = (work + tpb - 1) / tpb;
    if (b < 1) b = 1;
    if (b > kReduceMaxBlocks) b = kReduceMaxBlocks;
    return (unsigned)b;
}

}  // namespace

template <typename R>
void launch_pbb_step(const Lat<R, R>& src, const Lat<R, R>& dst, const Geo& g, const Phys<R>& ph, const R* ns,
                     const int32_t* ns_list, int64_t ns_count, const Reduce& red, double* series, int64_t cap,
                     int64_t* d_itime, cudaStream_t st) {
    if (series) {  // the force first: it reads the source lattice the step leaves unchanged
        k_pbb_force<R><<<capped_grid(ns_count, 256), 256, 0, st>>>(src, g, ns, ns_list, ns_count, red, series, cap,
                                                                    d_itime);
    }
    if constexpr (sizeof(R) == 4) {
        bool aligned = true;
        for (int q = 0; q < Q; ++q)
            aligned = aligned && reinterpret_cast<uintptr_t>(src.pop[q]) % 8 == 0 &&
                      reinterpret_cast<uintptr_t>(dst.pop[q]) % 8 == 0;
        if (g.l % 2 == 0 && aligned && reinterpret_cast<uintptr_t>(ns) % 8 == 0) {
            const int np = g.l / 2;
            dim3 grid((np + 127) / 128, g.m, g.n);
            k_pbb_pair<5><<<grid, 128, 0, st>>>(src, dst, g, ph, ns, np);
            return;
        }
    }
    k_pbb_step<R><<<capped_grid(g.N, 256), 256, 0, st>>>(src, dst, g, ph, ns);
}

template <typename R>
void launch_pbb_adjoint(const Lat<R, R>& f, const Geo& g, const Phys<R>& ph, const R* ns, const Lat<R, R>& lam_in,
                        const Lat<R, R>& lam_out, R* gmu, double* grad, R gamma, const HaloAdjointDevice& t,
                        cudaStream_t st) {
    // resident blocks of 256 per SM the registers are sized for: FP32 3 (80 registers), FP64 2
    k_pbb_adjoint<R, sizeof(R) == 4 ? 3 : 2><<<capped_grid(g.N, 256), 256, 0, st>>>(f, g, ph, ns, lam_in, lam_out,
                                                                                      gmu, grad, gamma);
    if (t.ncopy > 0)
        k_adj_copy<R><<<(unsigned)((t.ncopy + 255) / 256), 256, 0, st>>>(g, t.copy_key, t.copy_start, t.copy_slot,
                                                                          t.ncopy, gmu, lam_out);
    if (t.nout > 0)
        k_adj_outflow<R><<<(unsigned)((t.nout + 255) / 256), 256, 0, st>>>(g, t.out_jk, t.out_start, t.out_slot,
                                                                            t.out_q, t.nout, gmu, f, lam_out);
}

template void launch_pbb_step<float>(const Lat<float, float>&, const Lat<float, float>&, const Geo&,
                                     const Phys<float>&, const float*, const int32_t*, int64_t, const Reduce&,
                                     double*, int64_t, int64_t*, cudaStream_t);
template void launch_pbb_step<double>(const Lat<double, double>&, const Lat<double, double>&, const Geo&,
                                      const Phys<double>&, const double*, const int32_t*, int64_t, const Reduce&,
                                      double*, int64_t, int64_t*, cudaStream_t);
template void launch_pbb_adjoint<float>(const Lat<float, float>&, const Geo&, const Phys<float>&, const float*,
                                        const Lat<float, float>&, const Lat<float, float>&, float*, double*, float,
                                        const HaloAdjointDevice&, cudaStream_t);
template void launch_pbb_adjoint<double>(const Lat<double, double>&, const Geo&, const Phys<double>&,
                                         const double*, const Lat<double, double>&, const Lat<double, double>&,
                                         double*, double*, double, const HaloAdjointDevice&, cudaStream_t);

}  // namespace eup
