// step2d_pair.cuh -- one launch per RK4 step of 2-D Cahn-Hilliard on grids
// whose four sides are periodic, with every thread advancing two x-adjacent
// cells at a time.
//
// Same tile scheme as step2d.cuh (u on the tile + E loaded once, the four
// stages in shared memory on regions shrinking by H per stage), arranged for
// issue efficiency:
//   * cells are processed as pairs: FP32 arithmetic uses the packed f32x2
//     instructions of sm_100 (fma/add/mul .rn on both lanes, each lane
//     rounded exactly as the scalar instruction), shared memory is read and
//     written 8 (FP32) or 16 (FP64) bytes at a time;
//   * each thread owns one pair column and a block of consecutive rows, so a
//     5-point stencil keeps its north / centre / south pairs in registers and
//     loads one pair plus the two side neighbours per row;
//   * the k pass of stage s writes y_{s+1} = u + a k_s straight into the
//     stage-state array (the CH k pass reads mu only) and folds k_s into the
//     RK4 sum of the tile cells, so a stage is two passes and two barriers.
// Regions are rounded outward to whole pairs; the extra cells read only
// in-bounds shared memory and are never used by a cell that is kept.
// Temporal blocking (depth NS = 2): u is loaded on the tile + 16, the first
// step's four stages run on regions 8 cells wider and its update (tile + 8)
// is written back into shared memory, then the second step runs as usual: two
// time steps per launch and per pass over HBM, at the cost of the wider
// regions' recomputation.
// Every cell sees the scalar path's operations in the scalar path's order
// (Equation.cu:65-76 for the Laplacian, the CH driver's mu and rhs, the RK4
// combination of Solver.cu), so the bits equal those of step_box / stage_box.
#pragma once

#include <cuda_runtime.h>

#include "step2d.cuh"

namespace phix {

// ---- pairs of cells -------------------------------------------------------
template <typename T> struct PairOf;
template <> struct PairOf<float> { using V = float2; };
template <> struct PairOf<double> { using V = double2; };

__device__ __forceinline__ float2 p_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 p_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 p_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// a - b rounded once: b * (-1) is exact, so fma(b, -1, a) = fl(a - b) on each lane
__device__ __forceinline__ float2 p_sub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 p_splat(float v) { return make_float2(v, v); }

__device__ __forceinline__ double2 p_add(double2 a, double2 b) { return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y)); }
__device__ __forceinline__ double2 p_mul(double2 a, double2 b) { return make_double2(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)); }
__device__ __forceinline__ double2 p_fma(double2 a, double2 b, double2 c) {
    return make_double2(__fma_rn(a.x, b.x, c.x), __fma_rn(a.y, b.y, c.y));
}
__device__ __forceinline__ double2 p_sub(double2 a, double2 b) { return make_double2(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y)); }
__device__ __forceinline__ double2 p_splat(double v) { return make_double2(v, v); }

template <typename T>
__device__ __forceinline__ typename PairOf<T>::V p_ld(const T* p) {
    return *reinterpret_cast<const typename PairOf<T>::V*>(p);
}
template <typename T>
__device__ __forceinline__ void p_st(T* p, typename PairOf<T>::V v) {
    *reinterpret_cast<typename PairOf<T>::V*>(p) = v;
}

// 5-point Laplacian of the pair c from its west, east, north (row - 1) and
// south (row + 1) neighbour pairs (tile_lap: v2 = 2c; t = (f+ - v2) + f-;
// v = tx*i2x; v = fma(ty, i2y, v)).  Returns v and leaves 2c in *v2.
template <class V>
__device__ __forceinline__ V p_lap(V c, V north, V south, V west, V east, V i2x, V i2y, V* v2) {
    *v2 = p_add(c, c);  // 2*c: exact, equal to rmul(2, c)
    const V tx = p_add(p_sub(east, *v2), west);
    const V ty = p_add(p_sub(south, *v2), north);
    return p_fma(ty, i2y, p_mul(tx, i2x));
}

// mu and the right-hand side of a pair through a stage policy: lane by lane
// (any policy, e.g. the C++ DSL's PolUser with the user's functor), or, for
// the built-in PolCH, in the packed forms below.  Both round every lane as the
// scalar policy does.
template <typename T, class Pol>
struct PairPolicy {
    using V = typename PairOf<T>::V;
    __device__ static __forceinline__ V mu(const StageArgs<T>& S, const Pol& pol, V c, V lap, V) {
        return V{pol.mu(S, c.x, lap.x, (T)0), pol.mu(S, c.y, lap.y, (T)0)};
    }
    __device__ static __forceinline__ V rhs(const StageArgs<T>& S, const Pol& pol, V lapmu, V c) {
        T kx[2], ky[2];
        pol.rhs(S, lapmu.x, c.x, (T)0, (T)0, (T)0, kx);
        pol.rhs(S, lapmu.y, c.y, (T)0, (T)0, (T)0, ky);
        return V{kx[0], ky[0]};
    }
};

template <typename T>
struct PairPolicy<T, PolCH> {
    using V = typename PairOf<T>::V;
    __device__ static __forceinline__ V mu(const StageArgs<T>& S, const PolCH&, V c, V lap, V v2) {
        const V two_rho = p_splat(S.p[2]), ca = p_splat(S.p[3]), cb = p_splat(S.p[4]);
        const V mk = p_splat(S.p[1]), one = p_splat((T)1), zero = p_splat((T)0);
        // f'(c) = (two_rho (c - ca)) (c - cb) ((2c - ca) - cb)   (f_dw)
        const V fa = p_mul(p_mul(two_rho, p_sub(c, ca)), p_sub(c, cb));
        const V fd = p_mul(fa, p_sub(p_sub(v2, ca), cb));
        // mu = (-kappa) lap + (1 f' + 0)   (PolCH::mu)
        return p_fma(mk, lap, p_fma(one, fd, zero));
    }
    __device__ static __forceinline__ V rhs(const StageArgs<T>& S, const PolCH&, V lapmu, V) {
        return p_fma(p_splat(S.p[0]), lapmu, p_splat((T)0));  // k = M lap(mu) + 0
    }
};

// Tile geometry: NS = time steps per launch (temporal-block depth 1 or 2).
// u is loaded on the tile + E, E = 8 NS; each RK4 step shrinks the computed
// regions by 8.  With NS = 2 the first step's update covers the tile + 8
// (EO), written back into U (and, FP32, the low parts into LO) for the second.
template <typename T, int TX, int TY, int NRP, int NS = 1>
struct StepPair {
    static constexpr int TX_ = TX, TY_ = TY, NRP_ = NRP, NS_ = NS;
    static constexpr int H = PolCH::H, E1 = 4 * H, E = E1 * NS, EO = E1 * (NS - 1);
    static constexpr int P = TX + 2 * E, R = TY + 2 * E;  // row pitch and rows of U, Y, M
    static constexpr int NC = P / 2;                      // pair columns
    static constexpr int NT = NC * NRP;                   // threads per CTA
    static constexpr int AX = TX + 2 * EO, AY = TY + 2 * EO;  // RK4 sum (and low parts) of the first update region
    static constexpr bool LO_SMEM = NS > 1 && sizeof(T) == 4;
    static_assert(NS == 1 || NS == 2, "temporal-block depth 1 or 2");
    static_assert(TX % 2 == 0 && E % 2 == 0, "pairs need an even tile width and halo");
    static constexpr size_t smem_bytes() {
        return sizeof(T) * ((size_t)3 * P * R + (size_t)AX * AY * (LO_SMEM ? 2 : 1));
    }
    // CTAs per SM that the shared memory admits (228 KB per SM, 1 KB reserved
    // per CTA), at most 2048 threads: the launch bound asks ptxas to keep
    // the registers within that many CTAs
    static constexpr int FIT = (int)((228 * 1024) / (smem_bytes() + 1024));
    static constexpr int MINB = FIT < 1 ? 1 : (FIT > 2048 / NT ? 2048 / NT : FIT);
};

// A pass over the region e: rows [LO, LO + RH) cut into NRP blocks of Q or
// Q + 1 consecutive rows (the first REM row phases take the longer blocks;
// thread row phase rp starts at r0(rp)), and the pair columns [PLO, PHI),
// the region's columns rounded out to whole pairs.  Each thread walks Q rows
// unconditionally plus at most one more, so the unrolled row loops carry no
// per-row exit tests.
template <int TX, int TY, int E, int NRP, int e>
struct PairRegion {
    static constexpr int LO = E - e, RH = TY + 2 * e, Q = RH / NRP, REM = RH % NRP;
    static constexpr int PLO = (E - e) >> 1, PHI = (E + TX + e + 1) >> 1;
    static_assert(Q >= 1, "fewer region rows than row blocks");
    __device__ static __forceinline__ int r0(int rp) { return LO + rp * Q + min(rp, REM); }
};

// Walks this thread's rows of the region with the 5-point window of `src`
// (north / centre / south pairs in registers, west and east scalars loaded),
// calling f(j, lap(src), centre pair, 2 * centre) for rows r0 + j.
template <typename T, class Rg, int P, class F>
__device__ __forceinline__ void pair_rows(const T* __restrict__ src, int rp, typename PairOf<T>::V i2x,
                                          typename PairOf<T>::V i2y, F&& f) {
    using V = typename PairOf<T>::V;
    V n = p_ld(src - P), c = p_ld(src);
    auto row = [&](int j) {
        const V s = p_ld(src + (j + 1) * P);
        const T w = src[j * P - 1], ee = src[j * P + 2];
        V v2;
        const V lap = p_lap(c, n, s, V{w, c.x}, V{c.y, ee}, i2x, i2y, &v2);
        f(j, lap, c, v2);
        n = c;
        c = s;
    };
#pragma unroll
    for (int j = 0; j < Rg::Q; ++j) row(j);
    if (Rg::REM && rp < Rg::REM) row(Rg::Q);
}

// One mu pass: M = mu(Y) on the region e (rounded to pairs).
template <typename T, class Pol, class G, int e>
__device__ __forceinline__ void pair_mu_pass(const StageArgs<T>& S, const Pol& pol, const T* __restrict__ Y,
                                             T* __restrict__ M, int pc, int rp) {
    using Rg = PairRegion<G::TX_, G::TY_, G::E, G::NRP_, e>;
    using V = typename PairOf<T>::V;
    constexpr int P = G::P;
    if (pc < Rg::PLO || pc >= Rg::PHI) return;
    const int off0 = Rg::r0(rp) * P + 2 * pc;
    T* m = M + off0;
    pair_rows<T, Rg, P>(Y + off0, rp, p_splat(S.i2[0]), p_splat(S.i2[1]), [&](int j, V lap, V c, V v2) {
        p_st(m + j * P, PairPolicy<T, Pol>::mu(S, pol, c, lap, v2));
    });
}

// One k pass (stages 1-3): k = rhs(lap mu) on the region e; Y = u + a k
// there; the RK4 sum (k1, then + 2 k2, + 2 k3) of the step's update region,
// the tile + EA, in ACC (row pitch TX + 2 EA).
template <typename T, class Pol, class G, int e, int STAGE, int EA>
__device__ __forceinline__ void pair_k_pass(const StageArgs<T>& S, const Pol& pol, const T* __restrict__ M,
                                            const T* __restrict__ U, T* __restrict__ Y, T* __restrict__ ACC, T a,
                                            int pc, int rp) {
    using Rg = PairRegion<G::TX_, G::TY_, G::E, G::NRP_, e>;
    using V = typename PairOf<T>::V;
    constexpr int P = G::P, E = G::E, TX = G::TX_, TY = G::TY_, AP = TX + 2 * EA, A0 = E - EA;
    if (pc < Rg::PLO || pc >= Rg::PHI) return;
    const int r0 = Rg::r0(rp);
    const int off0 = r0 * P + 2 * pc;
    const V av = p_splat(a), two = p_splat((T)2);
    const bool col_in = 2 * pc >= A0 && 2 * pc < E + TX + EA;
    T* acc0 = ACC + (r0 - A0) * AP + 2 * pc - A0;  // dereferenced on update-region rows only
    pair_rows<T, Rg, P>(M + off0, rp, p_splat(S.i2[0]), p_splat(S.i2[1]), [&](int j, V lap, V mu, V) {
        const V k = PairPolicy<T, Pol>::rhs(S, pol, lap, mu);
        const int off = off0 + j * P;
        p_st(Y + off, p_fma(av, k, p_ld(U + off)));
        const int row = r0 + j;
        if (col_in && row >= A0 && row < E + TY + EA) {
            T* acc = acc0 + j * AP;
            p_st(acc, STAGE == 1 ? k : p_add(p_ld(acc), p_mul(two, k)));
        }
    });
}

// The four stages of one RK4 step in shared memory whose update region is the
// tile + EA: on return M holds mu of stage 4 on the tile + EA + 1 and ACC the
// sum k1 + 2 k2 + 2 k3 there (the update itself is the caller's pass).
template <typename T, class Pol, class G, int EA>
__device__ __forceinline__ void pair_four_stages(const StepArgs<T>& A, const Pol& pol, const T* __restrict__ U,
                                                 T* __restrict__ Y, T* __restrict__ M, T* __restrict__ ACC, int pc,
                                                 int rp) {
    constexpr int H = G::H;
    const StageArgs<T>& S = A.S;
    // stage 1: y1 = u
    pair_mu_pass<T, Pol, G, EA + 3 * H + 1>(S, pol, U, M, pc, rp);
    __syncthreads();
    pair_k_pass<T, Pol, G, EA + 3 * H, 1, EA>(S, pol, M, U, Y, ACC, A.dt2, pc, rp);
    __syncthreads();
    // stage 2
    pair_mu_pass<T, Pol, G, EA + 2 * H + 1>(S, pol, Y, M, pc, rp);
    __syncthreads();
    pair_k_pass<T, Pol, G, EA + 2 * H, 2, EA>(S, pol, M, U, Y, ACC, A.dt2, pc, rp);
    __syncthreads();
    // stage 3
    pair_mu_pass<T, Pol, G, EA + H + 1>(S, pol, Y, M, pc, rp);
    __syncthreads();
    pair_k_pass<T, Pol, G, EA + H, 3, EA>(S, pol, M, U, Y, ACC, A.dt, pc, rp);
    __syncthreads();
    // stage 4
    pair_mu_pass<T, Pol, G, EA + 1>(S, pol, Y, M, pc, rp);
    __syncthreads();
}

// u on the tile + E (periodic images of out-of-domain cells) into U (row
// pitch P, R rows): this thread's pair column on rows rp, rp + NRP, ...; all
// loads are issued before the first shared-memory store.  `inside`: the tile
// + E lies in the grid, so no image mapping is needed.
template <typename T, int E, int P, int R, int NRP>
__device__ __forceinline__ void pair_load_tile(const StageArgs<T>& S, T* __restrict__ U, int x0, int y0, int pc,
                                               int rp, bool inside) {
    using V = typename PairOf<T>::V;
    const Layout& L = S.L;
    constexpr int NLD = (R + NRP - 1) / NRP;
    V v[NLD];
    const int px = x0 - E + 2 * pc;
#pragma unroll
    for (int i = 0; i < NLD; ++i) {
        const int ly = rp + i * NRP, py = y0 - E + ly;
        if (ly < R) {
            if (inside) {
                const T* g = S.u[0] + L.origin + px + L.s[1] * py;
                v[i] = V{__ldg(g), __ldg(g + 1)};
            } else {
                int i0, i1;
                double cval;
                map3<2>(L, px, py, 0, &i0, &cval);  // periodic only: never MAP_CONST
                map3<2>(L, px + 1, py, 0, &i1, &cval);
                v[i] = V{__ldg(S.u[0] + i0), __ldg(S.u[0] + i1)};
            }
        }
    }
#pragma unroll
    for (int i = 0; i < NLD; ++i) {
        const int ly = rp + i * NRP;
        if (ly < R) p_st(U + ly * P + 2 * pc, v[i]);
    }
}

// The low parts of the compensated state at this thread's cells of the tile
// pass (region R0: rows fr0 + j, pair at x = gx), zero where there are none.
template <typename T, class R0, int E>
__device__ __forceinline__ void pair_lo_prefetch(const StageArgs<T>& S, typename PairOf<T>::V* lo_pf, int y0, int fr0,
                                                 int gx, bool fcol, bool x1, int rp) {
    const Layout& L = S.L;
#pragma unroll
    for (int j = 0; j <= R0::Q; ++j) {
        lo_pf[j] = p_splat((T)0);
        const int py = y0 + fr0 + j - E;
        if (S.ulo[0] && fcol && (j < R0::Q || rp < R0::REM) && py < L.n[1] && gx < L.n[0]) {
            const T* g = S.ulo[0] + L.origin + gx + L.s[1] * py;
            lo_pf[j].x = __ldg(g);
            if (x1) lo_pf[j].y = __ldg(g + 1);
        }
    }
}

// The low parts of the compensated state on the tile + EO (periodic images)
// into LO (row pitch AX): the first update of a depth-2 launch needs them.
template <typename T, class G>
__device__ __forceinline__ void pair_load_lo(const StageArgs<T>& S, T* __restrict__ LO, int x0, int y0, bool inside) {
    const Layout& L = S.L;
    constexpr int AX = G::AX, AY = G::AY, EO = G::EO;
    for (int i = threadIdx.x; i < AX * AY; i += G::NT) {
        const int px = x0 - EO + i % AX, py = y0 - EO + i / AX;
        int idx;
        double cval;
        if (inside) idx = L.origin + px + L.s[1] * py;
        else map3<2>(L, px, py, 0, &idx, &cval);  // periodic only: never MAP_CONST
        LO[i] = S.ulo[0] ? __ldg(S.ulo[0] + idx) : (T)0;
    }
}

// The first update of a depth-2 launch, on the tile + EO: u' = u + dt/6 sum
// (FP32: the compensated two-sum with the low parts in LO), written back into
// U and LO in place (each cell reads only its own u, lo and sum here).
template <typename T, class Pol, class G>
__device__ __forceinline__ void pair_mid_update(const StepArgs<T>& A, const Pol& pol, T* __restrict__ U,
                                                const T* __restrict__ M, const T* __restrict__ ACC,
                                                T* __restrict__ LO, int pc, int rp) {
    using Rg = PairRegion<G::TX_, G::TY_, G::E, G::NRP_, G::EO>;
    using V = typename PairOf<T>::V;
    constexpr int P = G::P, AP = G::AX, A0 = G::E - G::EO;
    const StageArgs<T>& S = A.S;
    if (pc < Rg::PLO || pc >= Rg::PHI) return;
    const int r0 = Rg::r0(rp);
    const int off0 = r0 * P + 2 * pc;
    const V dtf = p_splat(S.dtf);
    pair_rows<T, Rg, P>(M + off0, rp, p_splat(S.i2[0]), p_splat(S.i2[1]), [&](int j, V lap, V mu, V) {
        const V k = PairPolicy<T, Pol>::rhs(S, pol, lap, mu);
        const int ai = (r0 + j - A0) * AP + 2 * pc - A0;
        const V sum = p_add(p_ld(ACC + ai), k);
        const int off = off0 + j * P;
        const V u = p_ld(U + off);
        if constexpr (G::LO_SMEM) {
            const V d = p_mul(dtf, sum);
            const V l = p_ld(LO + ai);
            T h0, l0, h1, l1;
            twosum_update(u.x, l.x, d.x, &h0, &l0);
            twosum_update(u.y, l.y, d.y, &h1, &l1);
            p_st(U + off, V{h0, h1});
            p_st(LO + ai, V{l0, l1});
        } else {
            p_st(U + off, p_fma(dtf, sum, u));
        }
    });
}

// Ghost faces of the new state beside a depth-2 tile (as box_ghosts writes
// them): the periodic images of the intermediate state, which the first update
// left in U / LO on the tile + EO.
template <typename T, class G>
__device__ __forceinline__ void pair_ghosts_smem(const StageArgs<T>& S, const T* __restrict__ U,
                                                 const T* __restrict__ LO, int x0, int y0) {
    const Layout& L = S.L;
    const int n0 = L.n[0], n1 = L.n[1], gl = L.ghost;
    constexpr int E = G::E, P = G::P, EO = G::EO, AX = G::AX, TX = G::TX_, TY = G::TY_;
    auto put = [&](int px, int py) {
        const int lx = px - x0, ly = py - y0, dst = L.origin + px + L.s[1] * py;
        S.out[0][dst] = U[(ly + E) * P + lx + E];
        if (S.ulo[0]) S.outlo[0][dst] = G::LO_SMEM ? LO[(ly + EO) * AX + lx + EO] : (T)0;
    };
    if (x0 == 0 || x0 + TX >= n0)
        for (int i = threadIdx.x; i < TY * gl; i += G::NT) {
            const int py = y0 + i / gl, l = 1 + i % gl;
            if (py >= n1) continue;
            if (x0 == 0) put(-l, py);
            if (x0 + TX >= n0) put(n0 - 1 + l, py);
        }
    if (y0 == 0 || y0 + TY >= n1)
        for (int i = threadIdx.x; i < TX * gl; i += G::NT) {
            const int px = x0 + i % TX, l = 1 + i / TX;
            if (px >= n0) continue;
            if (y0 == 0) put(px, -l);
            if (y0 + TY >= n1) put(px, n1 - 1 + l);
        }
}

template <typename T, class Pol, int TX, int TY, int NRP, int NS>
__device__ __forceinline__ void step_pair_tile(const StepArgs<T>& A, const Pol& pol, T* __restrict__ sm, int x0,
                                               int y0) {
    using G = StepPair<T, TX, TY, NRP, NS>;
    using V = typename PairOf<T>::V;
    constexpr int E = G::E, P = G::P, R = G::R, NC = G::NC;
    T* U = sm;
    T* Y = sm + P * R;
    T* M = sm + 2 * P * R;
    T* ACC = sm + 3 * P * R;
    T* LO = ACC + G::AX * G::AY;  // depth 2, FP32: low parts of the first update region
    const StageArgs<T>& S = A.S;
    const Layout& L = S.L;
    const int n0 = L.n[0], n1 = L.n[1];
    const int pc = threadIdx.x % NC, rp = threadIdx.x / NC;

    const bool inside = x0 - E >= 0 && x0 + TX + E <= n0 && y0 - E >= 0 && y0 + TY + E <= n1;
    pair_load_tile<T, E, P, R, NRP>(S, U, x0, y0, pc, rp, inside);
    if constexpr (G::LO_SMEM) pair_load_lo<T, G>(S, LO, x0, y0, inside);
    // the low parts of this thread's cells of the final update, fetched now
    // so that their latency hides behind the four stages (depth 1)
    using R0 = PairRegion<TX, TY, E, NRP, 0>;
    const int fr0 = R0::r0(rp);
    const int gx = x0 + 2 * pc - E;  // x of the pair's first cell in the final pass
    const bool fcol = pc >= R0::PLO && pc < R0::PHI, x1 = gx + 1 < n0;
    constexpr bool LO_STATE = sizeof(T) == 4;  // compensated state: FP32 steppers only
    constexpr bool LO_PF = LO_STATE && NS == 1;
    V lo_pf[LO_PF ? R0::Q + 1 : 1];
    if constexpr (LO_PF) pair_lo_prefetch<T, R0, E>(S, lo_pf, y0, fr0, gx, fcol, x1, rp);
    __syncthreads();

    if constexpr (NS == 2) {  // the first time step, on the tile + 8
        pair_four_stages<T, Pol, G, G::EO>(A, pol, U, Y, M, ACC, pc, rp);
        pair_mid_update<T, Pol, G>(A, pol, U, M, ACC, LO, pc, rp);
        __syncthreads();
    }
    pair_four_stages<T, Pol, G, 0>(A, pol, U, Y, M, ACC, pc, rp);

    // k4 on the tile, then u' = u + dt/6 (((k1 + 2 k2) + 2 k3) + k4)
    if (fcol) {
        const V dtf = p_splat(S.dtf);
        const int off0 = fr0 * P + 2 * pc;
        pair_rows<T, R0, P>(M + off0, rp, p_splat(S.i2[0]), p_splat(S.i2[1]), [&](int j, V lap, V mu, V) {
            const V k = PairPolicy<T, Pol>::rhs(S, pol, lap, mu);
            const int py = y0 + fr0 + j - E;
            if (py < n1 && gx < n0) {  // inside the grid (partial tiles)
                const V sum = p_add(p_ld(ACC + (fr0 + j - E) * TX + 2 * pc - E), k);
                const V u = p_ld(U + off0 + j * P);
                const int idx = L.origin + gx + L.s[1] * py;
                if (LO_STATE && S.ulo[0]) {
                    const V d = p_mul(dtf, sum);
                    V l;
                    if constexpr (LO_PF) l = lo_pf[j];
                    else if constexpr (G::LO_SMEM) l = p_ld(LO + (py - y0 + G::EO) * G::AX + gx - x0 + G::EO);
                    else l = p_splat((T)0);
                    twosum_update(u.x, l.x, d.x, &S.out[0][idx], &S.outlo[0][idx]);
                    if (x1) twosum_update(u.y, l.y, d.y, &S.out[0][idx + 1], &S.outlo[0][idx + 1]);
                } else {
                    const V o = p_fma(dtf, sum, u);
                    S.out[0][idx] = o.x;
                    if (x1) S.out[0][idx + 1] = o.y;
                }
            }
        });
    }
    if (!inside) {
        if constexpr (NS == 1) box_ghosts<T, 2, 1, TX, TY, G::NT>(S, x0, y0);
        else pair_ghosts_smem<T, G>(S, U, LO, x0, y0);
    }
}

template <typename T, class Pol, int TX, int TY, int NRP, int NS = 1>
__global__ void __launch_bounds__(StepPair<T, TX, TY, NRP, NS>::NT, StepPair<T, TX, TY, NRP, NS>::MINB)
    step_pair(const StepArgs<T> A, const Pol pol) {
    extern __shared__ __align__(16) unsigned char step_smem[];
    // launched as a programmatic dependent of the previous step (the C++
    // Solver's launches): let the next step's CTAs be scheduled once every CTA
    // of this one runs, and read nothing before the previous step's writes are
    // visible.  Both are no-ops for an ordinary launch.
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    step_pair_tile<T, Pol, TX, TY, NRP, NS>(A, pol, reinterpret_cast<T*>(step_smem), blockIdx.x * TX,
                                            blockIdx.y * TY);
}

// Many fields in one launch: one CTA per entry of the tile list.
template <typename T, int TX, int TY, int NRP, int NS = 1>
__global__ void __launch_bounds__(StepPair<T, TX, TY, NRP, NS>::NT, StepPair<T, TX, TY, NRP, NS>::MINB)
    step_pair_batched(const StepArgs<T>* __restrict__ args, const BatchTile* __restrict__ tiles) {
    extern __shared__ __align__(16) unsigned char step_smem[];
    const BatchTile bt = tiles[blockIdx.x];
    const StepArgs<T> a = args[bt.inst];
    step_pair_tile<T, PolCH, TX, TY, NRP, NS>(a, PolCH{}, reinterpret_cast<T*>(step_smem), bt.x0, bt.y0);
}

// Grids the pair kernels take: 2-D, four periodic sides (the policy must be a
// Cahn-Hilliard form: mu on the tile + 1, k = rhs(lap mu)).
inline bool step_pair_supported(const Layout& L, int dim) {
    if (dim != 2) return false;
    for (int i = 0; i < 4; ++i)
        if (L.bc[i] != PHIX_BC_PERIODIC) return false;
    return true;
}

}  // namespace phix
