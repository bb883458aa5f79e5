// step2d.cuh -- one launch per classical RK4 time step of a single-field 2-D
// problem (temporal fusion of the four stages of Solver::rk4AdvanceGPU,
// Solver.cu:193-259).
//
// A CTA owns a TX x TY tile of the new state.  It loads the old state u on
// the tile plus E = 4H cells (H = halo one stage needs: 1 for lap(y), 2 for
// lap(mu(y))), then runs the four stages in shared memory, each on a region
// H cells narrower than the one before:
//   stage s computes k_s on the tile + H(4-s)   (stage 4: the tile itself)
//   y_{s+1} = u + a_s k_s on the tile + H(4-s)  (a = dt/2, dt/2, dt)
// and finally u' = u + dt/6 (((k1 + 2k2) + 2k3) + k4) on the tile.  Every
// value is computed by the same per-cell functions, in the same order, as the
// one-launch-per-stage kernels of stage.cuh, so the result is the same to the
// last bit; cells near the tile edge are computed by several CTAs.
//
// Boundaries: periodic and zero-flux.  Periodic halo cells are computed like
// any other cell from the wrapped u (the computation is translation
// invariant, so they equal the values at the wrapped cells).  Past a zero-flux
// side, y and mu are taken from the boundary cell (the ghost fill of
// NoFluxBC, Boundary.cu:129-160, and the clamped mu of lap(expr, bcs)); k is
// never needed there.  Dirichlet sides and sides without a BC use the
// per-stage kernels.
//
// HBM traffic per cell-update: read u (+ the low part of a compensated FP32
// state), write u' (+ low part), i.e. 2w (4w compensated) instead of the 13w
// of one launch per stage; tile halos are re-read from L2.
#pragma once

#include "phix/detail/stage.cuh"

namespace phix {

template <typename T>
struct StepArgs {
    StageArgs<T> S;  // L, u[0], ulo[0], out[0], outlo[0], i2, p; S.dtf = dt/6
    T dt2, dt;       // stage-state coefficients dt/2 and dt
};

template <typename T, class Pol, int TX, int TY>
struct Step2D {
    static constexpr int H = Pol::H, E = 4 * H;
    static constexpr int P = TX + 2 * E, R = TY + 2 * E;  // smem pitch and rows
    static constexpr int NARR = Pol::MU ? 4 : 3;          // U, Y, K (+ M)
    static constexpr size_t smem_bytes() { return sizeof(T) * (size_t)NARR * P * R; }
};

// Calls f(lx, ly) for every cell of the tile-local square region that extends
// the tile by e cells on each side.
template <int TX, int TY, int E, int e, int NT, class F>
__device__ __forceinline__ void for_region(F&& f) {
    constexpr int RW = TX + 2 * e, RH = TY + 2 * e, N = RW * RH, IT = (N + NT - 1) / NT;
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int i = threadIdx.x + it * NT;
        if (it + 1 < IT || i < N) {
            const int ly = i / RW, lx = i - ly * RW;
            f(lx + E - e, ly + E - e);
        }
    }
}

template <typename T, class Pol, int TX, int TY, int NT>
__device__ __forceinline__ void step_tile(const StepArgs<T>& A, const Pol& pol, T* __restrict__ sm, int x0, int y0) {
    using G = Step2D<T, Pol, TX, TY>;
    constexpr int H = G::H, E = G::E, P = G::P, R = G::R;
    constexpr int NI = (TX * TY + NT - 1) / NT;  // tile cells per thread
    T* U = sm;
    T* Y = sm + P * R;
    T* K = sm + 2 * P * R;
    T* M = Pol::MU ? sm + 3 * P * R : nullptr;
    const StageArgs<T>& S = A.S;
    const Layout& L = S.L;
    const int n0 = L.n[0], n1 = L.n[1];

    // zero-flux clamp bounds in tile-local coordinates (none: unbounded)
    constexpr int FAR = 1 << 20;
    const int cxlo = L.bc[0] == PHIX_BC_NOFLUX ? E - x0 : -FAR;
    const int cxhi = L.bc[1] == PHIX_BC_NOFLUX ? n0 - 1 - x0 + E : FAR;
    const int cylo = L.bc[2] == PHIX_BC_NOFLUX ? E - y0 : -FAR;
    const int cyhi = L.bc[3] == PHIX_BC_NOFLUX ? n1 - 1 - y0 + E : FAR;
    auto src = [&](int lx, int ly) { return min(max(ly, cylo), cyhi) * P + min(max(lx, cxlo), cxhi); };

    // u on the tile + E (mapped by the BCs; the z ghost planes are never read)
    const bool inside = x0 - E >= 0 && x0 + TX + E <= n0 && y0 - E >= 0 && y0 + TY + E <= n1;
    for_region<TX, TY, E, E, NT>([&](int lx, int ly) {
        const int px = x0 - E + lx, py = y0 - E + ly;
        int idx;
        if (inside) {
            idx = L.origin + px + L.s[1] * py;
        } else {
            double cval;
            map3<2>(L, px, py, 0, &idx, &cval);  // periodic / zero-flux only: never MAP_CONST
        }
        U[ly * P + lx] = __ldg(S.u[0] + idx);
    });
    __syncthreads();

    T acc[NI];
    const T* y = U;
#pragma unroll
    for (int s = 1; s <= 4; ++s) {
        const int e = H * (4 - s);  // k region of this stage
        if (s > 1) {
            // y_s = u + a k_{s-1} on the k region of the previous stage
            const T a = s == 4 ? A.dt : A.dt2;
            auto ypass = [&](int lx, int ly) {
                const int q = src(lx, ly);
                Y[ly * P + lx] = rfma(a, K[q], U[q]);
            };
            if (s == 2) for_region<TX, TY, E, 3 * H, NT>(ypass);
            else if (s == 3) for_region<TX, TY, E, 2 * H, NT>(ypass);
            else for_region<TX, TY, E, H, NT>(ypass);
            // RK4 sum of the tile: ((k1 + 2k2) + 2k3) + k4
#pragma unroll
            for (int j = 0; j < NI; ++j) {
                const int i = threadIdx.x + j * NT;
                if (i < TX * TY) {
                    const T k = K[(i / TX + E) * P + i % TX + E];
                    acc[j] = s == 2 ? k : radd(acc[j], rmul((T)2, k));
                }
            }
            y = Y;
            __syncthreads();
        }
        if (Pol::MU) {
            // mu on the k region + 1 (past a zero-flux side: mu of the boundary cell)
            auto mpass = [&](int lx, int ly) {
                M[ly * P + lx] = compute_mu<T, Pol, 2, P>(S, pol, y, nullptr, nullptr, y, src(lx, ly));
            };
            if (s == 1) for_region<TX, TY, E, 3 * H + 1, NT>(mpass);
            else if (s == 2) for_region<TX, TY, E, 2 * H + 1, NT>(mpass);
            else if (s == 3) for_region<TX, TY, E, H + 1, NT>(mpass);
            else for_region<TX, TY, E, 1, NT>(mpass);
            __syncthreads();
        }
        if (s < 4) {
            auto kpass = [&](int lx, int ly) {
                const int off = ly * P + lx;
                T k[2];
                compute_rhs<T, Pol, 2, P, P>(S, pol, M, nullptr, nullptr, off, y, nullptr, nullptr, y, nullptr,
                                             nullptr, off, k);
                K[off] = k[0];
            };
            if (s == 1) for_region<TX, TY, E, 3 * H, NT>(kpass);
            else if (s == 2) for_region<TX, TY, E, 2 * H, NT>(kpass);
            else for_region<TX, TY, E, H, NT>(kpass);
            __syncthreads();
        }
        (void)e;
    }

    // stage 4 on the tile and the update
#pragma unroll
    for (int j = 0; j < NI; ++j) {
        const int i = threadIdx.x + j * NT;
        if (i >= TX * TY) break;
        const int lx = i % TX, ly = i / TX;
        const int px = x0 + lx, py = y0 + ly;
        if (px >= n0 || py >= n1) continue;
        const int off = (ly + E) * P + lx + E;
        T k[2];
        compute_rhs<T, Pol, 2, P, P>(S, pol, M, nullptr, nullptr, off, Y, nullptr, nullptr, Y, nullptr, nullptr, off,
                                     k);
        const T sum = radd(acc[j], k[0]);
        const int idx = L.origin + px + L.s[1] * py;
        const T u = U[off];
        if (S.ulo[0]) {
            twosum_update(u, __ldg(S.ulo[0] + idx), rmul(S.dtf, sum), &S.out[0][idx], &S.outlo[0][idx]);
        } else {
            S.out[0][idx] = rfma(S.dtf, sum, u);
        }
    }
    if (!inside) box_ghosts<T, 2, 1, TX, TY, NT>(S, x0, y0);
}

template <typename T, class Pol, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT) step_box(const StepArgs<T> A, const Pol pol) {
    extern __shared__ __align__(16) unsigned char step_smem[];
    step_tile<T, Pol, TX, TY, NT>(A, pol, reinterpret_cast<T*>(step_smem), blockIdx.x * TX, blockIdx.y * TY);
}

// Many fields in one launch: one CTA per entry of the tile list (a persistent
// loop over tiles makes ptxas spill this body heavily).
template <typename T, class Pol, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT) step_box_batched(const StepArgs<T>* __restrict__ args,
                                                       const BatchTile* __restrict__ tiles, const Pol pol) {
    extern __shared__ __align__(16) unsigned char step_smem[];
    const BatchTile bt = tiles[blockIdx.x];
    const StepArgs<T> a = args[bt.inst];
    step_tile<T, Pol, TX, TY, NT>(a, pol, reinterpret_cast<T*>(step_smem), bt.x0, bt.y0);
}

// True when the fused step supports this grid's boundaries (2-D, every side
// periodic or zero-flux).
inline bool step2d_supported(const Layout& L, int dim) {
    if (dim != 2) return false;
    for (int i = 0; i < 4; ++i)
        if (L.bc[i] != PHIX_BC_PERIODIC && L.bc[i] != PHIX_BC_NOFLUX) return false;
    return true;
}

}  // namespace phix
