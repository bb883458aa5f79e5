#pragma once
// step2d_pair_ms.cuh -- the multi-step Euler Cahn-Hilliard step (MODE_MULTISTEP
// of stage_box: mu, the STEADY field, is formed from c and written out; c, the
// TRANSIENT field, gets c + dt * rhs(lap mu)) in the pair layout of
// step2d_pair.cuh, for 2-D grids whose four sides are periodic.
//
// One launch per step.  Each CTA loads c on its tile + 2 once, forms mu on the
// tile + 1 in shared memory (two x-adjacent cells per thread, north / centre /
// south pairs in registers), then walks the tile once more for lap(mu), the
// Euler update and the mu output.  The reference runs this step as: BCs on c,
// mu = program(c) (STEADY), BCs on mu, rhs = M lap(mu), c += dt rhs
// (Solver.cu:317-340 with Cahn-Hillard_double-well.cu:84-106); every cell
// sees those operations in that order, so the bits equal stage_box's.
//
// The policy supplies mu and rhs (PolCH from the C ABI, the DSL's PolUser from
// the C++ Solver); PolCH takes the packed forms of step_pair, any other policy
// is called lane by lane.

#include "phix/detail/step2d_pair.cuh"

namespace phix {

template <typename T, int TX, int TY, int NRP>
struct MsPair {
    static constexpr int E = 2;                           // c on the tile + 2, mu on the tile + 1
    static constexpr int P = TX + 2 * E, R = TY + 2 * E;  // row pitch and rows of U and M
    static constexpr int NC = P / 2;                      // pair columns
    static constexpr int NT = NC * NRP;                   // threads per CTA
    static_assert(TX % 2 == 0, "pairs need an even tile width");
    static_assert(NT <= 1024, "more threads than a CTA may have");
    static constexpr size_t smem_bytes() { return sizeof(T) * (size_t)2 * P * R; }
    // CTAs per SM that the shared memory admits (228 KB per SM, 1 KB reserved
    // per CTA), at most 2048 threads, and at least 48 registers a thread
    // (registers are granted per whole warp)
    static constexpr int FIT = (int)((228 * 1024) / (smem_bytes() + 1024));
    static constexpr int WARPS = (NT + 31) / 32;
    static constexpr int BY_THREADS = 64 / WARPS, BY_REGS = 65536 / (WARPS * 32 * 48);
    static constexpr int MINB0 = FIT < BY_THREADS ? FIT : BY_THREADS;
    static constexpr int MINB1 = MINB0 < BY_REGS ? MINB0 : BY_REGS;
    static constexpr int MINB = MINB1 < 1 ? 1 : MINB1;
};

template <typename T, class Pol, int TX, int TY, int NRP>
__device__ __forceinline__ void ms_pair_tile(const StageArgs<T>& S, const Pol& pol, T* __restrict__ sm, int x0,
                                             int y0) {
    using G = MsPair<T, TX, TY, NRP>;
    using V = typename PairOf<T>::V;
    using PP = PairPolicy<T, Pol>;
    constexpr int E = G::E, P = G::P, R = G::R, NC = G::NC;
    T* U = sm;
    T* M = sm + P * R;
    const Layout& L = S.L;
    const int n0 = L.n[0], n1 = L.n[1];
    const int pc = threadIdx.x % NC, rp = threadIdx.x / NC;
    const V i2x = p_splat(S.i2[0]), i2y = p_splat(S.i2[1]);

    const bool inside = x0 - E >= 0 && x0 + TX + E <= n0 && y0 - E >= 0 && y0 + TY + E <= n1;
    pair_load_tile<T, E, P, R, NRP>(S, U, x0, y0, pc, rp, inside);
    using R0 = PairRegion<TX, TY, E, NRP, 0>;
    const int fr0 = R0::r0(rp);
    const int gx = x0 + 2 * pc - E;  // x of the pair's first cell in the tile pass
    const bool fcol = pc >= R0::PLO && pc < R0::PHI, x1 = gx + 1 < n0;
    constexpr bool LO_STATE = sizeof(T) == 4;  // compensated state: FP32 steppers only
    V lo_pf[LO_STATE ? R0::Q + 1 : 1];
    if constexpr (LO_STATE) pair_lo_prefetch<T, R0, E>(S, lo_pf, y0, fr0, gx, fcol, x1, rp);
    else lo_pf[0] = p_splat((T)0);  // never read: plain state
    __syncthreads();

    // mu on the tile + 1
    {
        using R1 = PairRegion<TX, TY, E, NRP, 1>;
        if (pc >= R1::PLO && pc < R1::PHI) {
            const int off0 = R1::r0(rp) * P + 2 * pc;
            pair_rows<T, R1, P>(U + off0, rp, i2x, i2y,
                                [&](int j, V lap, V c, V v2) { p_st(M + off0 + j * P, PP::mu(S, pol, c, lap, v2)); });
        }
    }
    __syncthreads();

    // the tile: c' = c + dt rhs(lap mu), and mu written out
    if (fcol) {
        const V dtf = p_splat(S.dtf);
        const int off0 = fr0 * P + 2 * pc;
        pair_rows<T, R0, P>(M + off0, rp, i2x, i2y, [&](int j, V lap, V mu, V) {
            const int py = y0 + fr0 + j - E;
            if (py < n1 && gx < n0) {  // inside the grid (partial tiles)
                const V u = p_ld(U + off0 + j * P);
                const V k = PP::rhs(S, pol, lap, u);
                const int idx = L.origin + gx + L.s[1] * py;
                if (LO_STATE && S.ulo[0]) {
                    const V d = p_mul(dtf, k);
                    const V l = lo_pf[LO_STATE ? j : 0];
                    twosum_update(u.x, l.x, d.x, &S.out[0][idx], &S.outlo[0][idx]);
                    if (x1) twosum_update(u.y, l.y, d.y, &S.out[0][idx + 1], &S.outlo[0][idx + 1]);
                } else {
                    const V o = p_fma(dtf, k, u);
                    S.out[0][idx] = o.x;
                    if (x1) S.out[0][idx + 1] = o.y;
                }
                S.mu_out[idx] = mu.x;
                if (x1) S.mu_out[idx + 1] = mu.y;
            }
        });
    }

    if (!inside) {
        // ghost layer 1 of mu beside this tile (faces only, not corners): the
        // periodic images of mu, which the reference's BCs copy there before
        // the TRANSIENT step reads mu
        for (int i = threadIdx.x; i < TY; i += G::NT) {
            const int py = y0 + i;
            if (py >= n1) break;
            const int row = (i + E) * P;
            if (x0 == 0) S.mu_out[L.origin - 1 + L.s[1] * py] = M[row + E - 1];
            if (x0 + TX >= n0) S.mu_out[L.origin + n0 + L.s[1] * py] = M[row + E + n0 - x0];
        }
        for (int i = threadIdx.x; i < TX; i += G::NT) {
            const int px = x0 + i;
            if (px >= n0) break;
            if (y0 == 0) S.mu_out[L.origin + px - L.s[1]] = M[(E - 1) * P + E + i];
            if (y0 + TY >= n1) S.mu_out[L.origin + px + L.s[1] * n1] = M[(E + n1 - y0) * P + E + i];
        }
        box_ghosts<T, 2, 1, TX, TY, G::NT>(S, x0, y0);
    }
}

template <typename T, class Pol, int TX, int TY, int NRP>
__global__ void __launch_bounds__(MsPair<T, TX, TY, NRP>::NT, MsPair<T, TX, TY, NRP>::MINB)
    step_pair_ms(const StageArgs<T> A, const Pol pol) {
    extern __shared__ __align__(16) unsigned char step_smem[];
    ms_pair_tile<T, Pol, TX, TY, NRP>(A, pol, reinterpret_cast<T*>(step_smem), blockIdx.x * TX, blockIdx.y * TY);
}

}  // namespace phix
