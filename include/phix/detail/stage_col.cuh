// stage_col.cuh -- 2-D fused stage kernel with column-walking register
// blocking (same per-cell arithmetic as box_tile in stage.cuh, so the same
// bits).
//
// A CTA of TX x G threads owns a TX x TY tile; thread (cx, g) owns column cx
// within row group g (each phase's rows are split into G contiguous groups of
// a compile-time length).  A thread walks its column down its rows, keeping
// the previous, current and next values in registers, so a 5-point stencil
// costs three shared-memory reads (the row below comes from the walk, left
// and right from the neighbouring columns) and the index arithmetic is one
// add per row:
//   1. y = u + a k_prev on the tile + H (global loads, coalesced along x)
//   2. mu(y) on the tile + 1                   (policies with MU)
//   3. rhs(lap mu | y, lap y) on the tile, written as k or folded into the
//      final update.
// Tiles whose halo leaves the domain load y through the BC mapping; where mu
// would have to be clamped or set to a constant (a non-periodic side) the
// tile runs the generic box_tile instead.
#pragma once

#include "phix/detail/stage.cuh"

namespace phix {

template <typename T, class Pol, int TX, int TY>
struct ColSmem {
    static constexpr int H = Pol::H, NF = Pol::NF;
    static constexpr int WX = TX + 2 * H, WY = TY + 2 * H;  // y tile
    static constexpr int MX = TX + 2, MY = TY + 2;          // mu tile
    static constexpr size_t bytes() {
        return sizeof(T) * ((size_t)NF * WX * WY + (Pol::MU ? (size_t)MX * MY : 0));
    }
};

// Is mu needed past a non-periodic side for this tile?  (then: generic path)
__device__ __forceinline__ bool col_mu_simple(const Layout& L, int x0, int y0, int TX, int TY) {
    if (x0 - 1 < 0 && L.bc[0] != PHIX_BC_PERIODIC) return false;
    if (x0 + TX + 1 > L.n[0] && L.bc[1] != PHIX_BC_PERIODIC) return false;
    if (y0 - 1 < 0 && L.bc[2] != PHIX_BC_PERIODIC) return false;
    if (y0 + TY + 1 > L.n[1] && L.bc[3] != PHIX_BC_PERIODIC) return false;
    return true;
}

template <typename T, class Pol, int MODE, int TX, int TY, int G>
__device__ __forceinline__ void col_tile(const StageArgs<T>& A, const Pol& pol, T* __restrict__ sm, int x0, int y0) {
    static_assert(!Pol::MU || Pol::H >= 2, "mu needs a halo of 2");
    static_assert(TX % 32 == 0 && TX >= 2 * Pol::H, "whole warps per row group, halo columns from the first lanes");
    static_assert(TY % G == 0, "every row group owns output rows");
    static_assert(MODE != MODE_MULTISTEP, "the multi-step form runs box_tile");
    using S = ColSmem<T, Pol, TX, TY>;
    constexpr int H = S::H, NF = S::NF, WX = S::WX, WY = S::WY, MX = S::MX, MY = S::MY;
    constexpr int NT = TX * G;
    T* ys0 = sm;
    T* ys1 = sm + (NF > 1 ? WX * WY : 0);
    T* ms = sm + NF * WX * WY;
    const Layout& L = A.L;
    const int n0 = L.n[0], n1 = L.n[1];
    const int cx = threadIdx.x % TX, g = threadIdx.x / TX;
    const bool interior = x0 - H >= 0 && x0 + TX + H <= n0 && y0 - H >= 0 && y0 + TY + H <= n1;

    // ---- 1. stage state on the tile + H: column cx (and TX + cx for the 2H
    //         halo columns), the rows of this group ------------------------------
    {
        constexpr int PER = (WY + G - 1) / G;  // compile-time trip count: the loads issue back to back
        const int r0 = g * PER;
#pragma unroll
        for (int pass = 0; pass < 2; ++pass) {
            const int lx = pass == 0 ? cx : TX + cx;
            if (pass == 1 && cx >= 2 * H) break;
            const int px = x0 - H + lx;
            if (interior) {
                const int idx0 = L.origin + px + L.s[1] * (y0 - H + r0);
#pragma unroll
                for (int q = 0; q < PER; ++q) {
                    if (r0 + q < WY) {
                        const int idx = idx0 + q * L.s[1];
#pragma unroll
                        for (int f = 0; f < NF; ++f) {
                            T u = __ldg(A.u[f] + idx);
                            if (A.kin[f]) u = rfma(A.a, __ldg(A.kin[f] + idx), u);
                            (f == 0 ? ys0 : ys1)[(r0 + q) * WX + lx] = u;
                        }
                    }
                }
            } else {
#pragma unroll
                for (int q = 0; q < PER; ++q) {
                    if (r0 + q < WY) {
#pragma unroll
                        for (int f = 0; f < NF; ++f)
                            (f == 0 ? ys0 : ys1)[(r0 + q) * WX + lx] =
                                load_y<T, 2>(A, f, px, y0 - H + r0 + q, 0, false);
                    }
                }
            }
        }
    }
    __syncthreads();

    if (Pol::MU && !interior && !col_mu_simple(L, x0, y0, TX, TY)) {
        // a clamped or constant mu ring: the generic tile (re-loads y itself)
        __syncthreads();
        BoxSmem<T, Pol, 2, TX, TY>* bs = reinterpret_cast<BoxSmem<T, Pol, 2, TX, TY>*>(sm);
        box_tile<T, Pol, 2, MODE, TX, TY, NT>(A, pol, *bs, x0, y0);
        return;
    }

    // ---- 2. mu on the tile + 1 ------------------------------------------------
    if (Pol::MU) {
        constexpr int PER = (MY + G - 1) / G;
        const int r0 = g * PER;
#pragma unroll
        for (int pass = 0; pass < 2; ++pass) {
            const int mx = pass == 0 ? cx : TX + cx;  // mu column; y column = mx + H - 1
            if (pass == 1 && cx >= 2) break;
            if (r0 >= MY) break;
            const T* col = ys0 + (mx + H - 1);
            T a = col[(r0 + H - 2) * WX];  // y row above mu row r0
            T b = col[(r0 + H - 1) * WX];
#pragma unroll
            for (int q = 0; q < PER; ++q) {
                const int mr = r0 + q;
                if (mr >= MY) break;
                const int yr = mr + H - 1;
                const T c = col[(yr + 1) * WX];
                const T l = col[yr * WX - 1], r = col[yr * WX + 1];
                const T b2 = rmul((T)2, b);
                const T lap = lap_combine<T, 2>(second_diff(r, b2, l), second_diff(c, b2, a), (T)0, A.i2[0], A.i2[1],
                                                A.i2[2]);
                const T other = NF > 1 ? ys1[yr * WX + mx + H - 1] : (T)0;
                ms[mr * MX + mx] = pol.mu(A, b, lap, other);
                a = b;
                b = c;
            }
        }
        __syncthreads();
    }

    // ---- 3. right-hand side and output: column cx, the rows of this group ----
    {
        constexpr int PER = TY / G;
        const int r0 = g * PER;
        const int px = x0 + cx;
        const bool colok = px < n0;
        const T* mcol = ms + (cx + 1);
        const T* y0c = ys0 + (cx + H);
        const T* y1c = ys1 + (cx + H);
        T ma = Pol::MU ? mcol[r0 * MX] : (T)0, mb = Pol::MU ? mcol[(r0 + 1) * MX] : (T)0;
        T ya = Pol::LAP_Y0 ? y0c[(r0 + H - 1) * WX] : (T)0, yb = y0c[(r0 + H) * WX];
        T za = Pol::LAP_Y1 ? y1c[(r0 + H - 1) * WX] : (T)0, zb = NF > 1 ? y1c[(r0 + H) * WX] : (T)0;
        const int idx0 = L.origin + px + L.s[1] * (y0 + r0);
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            const int r = r0 + q;
            const int idx = idx0 + q * L.s[1];
            T lapmu = (T)0, lapy0 = (T)0, lapy1 = (T)0;
            if (Pol::MU) {
                const T mc = mcol[(r + 2) * MX];
                const T ml = mcol[(r + 1) * MX - 1], mr = mcol[(r + 1) * MX + 1];
                const T m2 = rmul((T)2, mb);
                lapmu = lap_combine<T, 2>(second_diff(mr, m2, ml), second_diff(mc, m2, ma), (T)0, A.i2[0], A.i2[1],
                                          A.i2[2]);
                ma = mb;
                mb = mc;
            }
            const int yr = r + H;
            const T ync = y0c[(yr + 1) * WX];
            if (Pol::LAP_Y0) {
                const T yl = y0c[yr * WX - 1], yrr = y0c[yr * WX + 1];
                const T y2 = rmul((T)2, yb);
                lapy0 = lap_combine<T, 2>(second_diff(yrr, y2, yl), second_diff(ync, y2, ya), (T)0, A.i2[0],
                                          A.i2[1], A.i2[2]);
            }
            T znc = (T)0;
            if (NF > 1) {
                znc = y1c[(yr + 1) * WX];
                if (Pol::LAP_Y1) {
                    const T zl = y1c[yr * WX - 1], zr = y1c[yr * WX + 1];
                    const T z2 = rmul((T)2, zb);
                    lapy1 = lap_combine<T, 2>(second_diff(zr, z2, zl), second_diff(znc, z2, za), (T)0, A.i2[0],
                                              A.i2[1], A.i2[2]);
                }
            }
            T k[2];
            pol.rhs(A, lapmu, yb, lapy0, zb, lapy1, k);
            if (colok && y0 + r < n1) {
#pragma unroll
                for (int f = 0; f < NF; ++f) emit<T, MODE>(A, f, idx, k[f]);
            }
            ya = yb;
            yb = ync;
            za = zb;
            zb = znc;
        }
    }

    if (MODE != MODE_K && !interior) box_ghosts<T, 2, NF, TX, TY, NT>(A, x0, y0);
}

template <typename T, class Pol, int MODE, int TX, int TY, int G>
__global__ void __launch_bounds__(TX * G) stage_col(const StageArgs<T> A, const Pol pol) {
    extern __shared__ __align__(16) unsigned char col_smem[];
    col_tile<T, Pol, MODE, TX, TY, G>(A, pol, reinterpret_cast<T*>(col_smem), blockIdx.x * TX, blockIdx.y * TY);
}

// Shared memory a stage_col launch needs (it also hosts box_tile's smem for
// tiles that fall back to the generic path).
template <typename T, class Pol, int TX, int TY>
constexpr size_t col_smem_bytes() {
    return ColSmem<T, Pol, TX, TY>::bytes() > sizeof(BoxSmem<T, Pol, 2, TX, TY>) ? ColSmem<T, Pol, TX, TY>::bytes()
                                                                                  : sizeof(BoxSmem<T, Pol, 2, TX, TY>);
}

}  // namespace phix
