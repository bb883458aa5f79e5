// stage.cuh -- fused Runge-Kutta / Euler stage kernels.
//
// One launch computes, for every physical cell of its tile,
//   y   = u + a * k_prev                 (kernel_rk4_tmp, Solver.cu:49-56)
//   ghost(y) by the field's BCs          (kernel_periodic/noflux/fixed, Boundary.cu:95-195)
//   rhs = Equation::computeRHS(y)        (Equation.cu:257-276, every DSL term)
// and writes either k_s = rhs (intermediate RK4 stage) or the new state
//   RK4  : u + dt/6 (k1 + 2k2 + 2k3 + k4)  (kernel_rk4_update, Solver.cu:61-71)
//   Euler: u + dt * rhs                    (kernel_axpy, Solver.cu:30-35)
// The BCs never run as kernels: halo cells of the tile are loaded from the
// mapped interior cell (periodic wrap, zero-flux clamp) or set to the Dirichlet
// value.  For lap(expr, bcs) (the Cahn-Hilliard biharmonic) the chemical
// potential mu is formed in shared memory on the tile plus one ring, with the
// same BC mapping applied to mu, so mu never touches HBM
// (makeStencilOnExprTerm, Equation.cu:537-594).
//
// Work per launch: 2D/1D use a TX x TY box tile per CTA; 3D uses a TX x TY
// in-plane tile that marches RZ planes along z with ring buffers of stage-state
// and mu planes, so every input plane is read once per stage.
#pragma once

#include "phix/detail/common.cuh"

namespace phix {

// MODE_MULTISTEP: the reference's multi-step Euler Cahn-Hilliard
// (Solver.cu:317-340 with Cahn-Hillard_double-well.cu:84-106): mu (STEADY) is
// the smem mu of the tile, written out as a field; c (TRANSIENT) gets the
// Euler update from M*lap(mu).
// MODE_RK4_STEP (C++ DSL launches only): the whole RK4 step in one launch
// (the pair kernel of step2d_pair.cuh), where the grid and term form allow.
enum : int { MODE_K = 0, MODE_RK4_FINAL = 1, MODE_EULER_FINAL = 2, MODE_MULTISTEP = 3, MODE_RK4_STEP = 4 };

template <typename T>
struct StageArgs {
    Layout L;
    const T* u[2];    // state at the start of the step
    const T* kin[2];  // previous stage k (nullptr in stage 1 / Euler)
    const T* k1[2];   // RK4 final stage only
    const T* k2[2];
    T* out[2];        // k_s, or the new state in the final modes
    T* mu_out;        // MODE_MULTISTEP: the STEADY mu field
    const T* ulo[2];  // compensated state: low parts of u (null = plain state)
    T* outlo[2];      // final modes with ulo: low parts of the new state
    T a;              // y = u + a * kin
    T dtf;            // dt/6 (RK4 final) or dt (Euler)
    T i2[3];          // 1/d^2 per axis
    T p[8];           // physics coefficients (make_coeffs in stepper.cu)
};

// ---------------------------------------------------------------------------
// Physics policies.  A policy fixes the number of fields NF, the halo H, whether
// a chemical potential mu (lap(expr, bcs)) is formed on tile+1 (MU), which
// Laplacians of the stage states the right-hand side needs (LAP_Y0, LAP_Y1),
// and computes, in the reference's term order,
//   mu(c, lap c, other field)                          (the inner expression)
//   rhs(lap mu, y0, lap y0, y1, lap y1) -> k[NF]         (the equation's terms)
// Built-in policies read their coefficients from StageArgs::p; policies
// carrying user functors (the C++ DSL) hold them as members.
// ---------------------------------------------------------------------------
struct PolAC {  // L*kappa*lap(phi) + L*pw(phi, p - p^3)
    static constexpr int NF = 1, H = 1;
    static constexpr bool MU = false, LAP_Y0 = true, LAP_Y1 = false;
    template <typename T>
    __device__ __forceinline__ T mu(const StageArgs<T>&, T, T, T) const { return (T)0; }
    template <typename T>
    __device__ __forceinline__ void rhs(const StageArgs<T>& A, T, T y0, T lapy0, T, T, T* k) const {
        k[0] = rfma(A.p[1], f_ac(y0), rfma(A.p[0], lapy0, (T)0));  // rhs = 0; += (L*kappa)*lap; += L*f
    }
};
struct PolCH {  // M*lap(pw(c, f') - kappa*lap(c), bcs)
    static constexpr int NF = 1, H = 2;
    static constexpr bool MU = true, LAP_Y0 = false, LAP_Y1 = false;
    template <typename T>
    __device__ __forceinline__ T mu(const StageArgs<T>& A, T c, T lapc, T) const {
        // scratch = 0; scratch += 1*f'(c); scratch += (-kappa)*lap(c)
        return rfma(A.p[1], lapc, rfma((T)1, f_dw(c, A.p[2], A.p[3], A.p[4]), (T)0));
    }
    template <typename T>
    __device__ __forceinline__ void rhs(const StageArgs<T>& A, T lapmu, T, T, T, T, T* k) const {
        k[0] = rfma(A.p[0], lapmu, (T)0);  // rhs = 0; rhs += M*lap(mu)
    }
};
struct PolCHAC {  // coupled (c, eta), see PHIX_PHYS_CHAC
    static constexpr int NF = 2, H = 2;
    static constexpr bool MU = true, LAP_Y0 = false, LAP_Y1 = true;
    template <typename T>
    __device__ __forceinline__ T mu(const StageArgs<T>& A, T c, T lapc, T e) const {
        return rfma(A.p[1], lapc, rfma((T)1, f_chac_c(c, e, A.p[4]), (T)0));
    }
    template <typename T>
    __device__ __forceinline__ void rhs(const StageArgs<T>& A, T lapmu, T y0, T, T y1, T lapy1, T* k) const {
        k[0] = rfma(A.p[0], lapmu, (T)0);
        // rhs = 0; rhs += (-L)*f_eta(eta, c); rhs += (L*kappa_eta)*lap(eta)
        k[1] = rfma(A.p[2], lapy1, rfma(A.p[3], f_chac_e(y1, y0, A.p[4]), (T)0));
    }
};

template <int PHYS> struct PolOf;
template <> struct PolOf<PHIX_PHYS_AC> { using type = PolAC; };
template <> struct PolOf<PHIX_PHYS_CH> { using type = PolCH; };
template <> struct PolOf<PHIX_PHYS_CHAC> { using type = PolCHAC; };

// ---------------------------------------------------------------------------
// per-cell helpers
// ---------------------------------------------------------------------------

// Flat stored index of (possibly out-of-domain) coordinates after BC mapping,
// or MAP_CONST with the constant the ghost fill would have written.
template <int DIM>
__device__ __forceinline__ int map3(const Layout& L, int px, int py, int pz, int* idx, double* cval) {
    int qx, qy = py, qz = pz;
    if (map_axis(px, L.n[0], L.bc[0], L.bc[1], L.bcv[0], L.bcv[1], L.ghost, &qx, cval) == MAP_CONST) return MAP_CONST;
    if (DIM >= 2 && map_axis(py, L.n[1], L.bc[2], L.bc[3], L.bcv[2], L.bcv[3], L.ghost, &qy, cval) == MAP_CONST)
        return MAP_CONST;
    if (DIM >= 3 && map_axis(pz, L.n[2], L.bc[4], L.bc[5], L.bcv[4], L.bcv[5], L.ghost, &qz, cval) == MAP_CONST)
        return MAP_CONST;
    *idx = L.origin + qx + L.s[1] * qy + L.s[2] * qz;
    return MAP_IN;
}

// Stage state of field f at (px,py,pz).
template <typename T, int DIM>
__device__ __forceinline__ T load_y(const StageArgs<T>& A, int f, int px, int py, int pz, bool interior) {
    int idx;
    if (interior) {
        idx = A.L.origin + px + A.L.s[1] * py + A.L.s[2] * pz;
    } else {
        double cval;
        if (map3<DIM>(A.L, px, py, pz, &idx, &cval) == MAP_CONST) return (T)cval;
    }
    T u = __ldg(A.u[f] + idx);
    if (A.kin[f] == nullptr) return u;
    return rfma(A.a, __ldg(A.kin[f] + idx), u);
}

// How mu is obtained at coordinate p along one axis: computed at p (inside or
// periodic), at the clamped cell (zero-flux), or a constant (Dirichlet value,
// 0 without BC: the scratch is zeroed and never written there).
__device__ __forceinline__ int mu_axis(int p, int n, int bc_lo, int bc_hi, double v_lo, double v_hi, int* q,
                                       double* cval) {
    if (p >= 0 && p < n) { *q = p; return MAP_IN; }
    int bc = p < 0 ? bc_lo : bc_hi;
    if (bc == PHIX_BC_PERIODIC) { *q = p; return MAP_IN; }
    if (bc == PHIX_BC_NOFLUX) { *q = p < 0 ? 0 : n - 1; return MAP_IN; }
    *cval = bc == PHIX_BC_FIXED ? (p < 0 ? v_lo : v_hi) : 0.0;
    return MAP_CONST;
}

// Laplacian at offset `off` of a tile plane `c` (pitch W) with z neighbours
// `m`, `p` (3-D).
template <typename T, int DIM, int W>
__device__ __forceinline__ T tile_lap(const StageArgs<T>& A, const T* c, const T* m, const T* p, int off) {
    const T v2 = rmul((T)2, c[off]);
    T tx = second_diff(c[off + 1], v2, c[off - 1]);
    T ty = DIM >= 2 ? second_diff(c[off + W], v2, c[off - W]) : (T)0;
    T tz = DIM >= 3 ? second_diff(p[off], v2, m[off]) : (T)0;
    return lap_combine<T, DIM>(tx, ty, tz, A.i2[0], A.i2[1], A.i2[2]);
}

// mu at tile-local offset `off` of y-plane `yc0` (planes `ym0`, `yp0` below and
// above in z for 3-D; `yc1` the second field).  W = row pitch of the y tile.
template <typename T, class Pol, int DIM, int W>
__device__ __forceinline__ T compute_mu(const StageArgs<T>& A, const Pol& pol, const T* yc0, const T* ym0,
                                        const T* yp0, const T* yc1, int off) {
    const T lap = tile_lap<T, DIM, W>(A, yc0, ym0, yp0, off);
    return pol.mu(A, yc0[off], lap, Pol::NF > 1 ? yc1[off] : (T)0);
}

// Right-hand side at a cell: `m*` are mu planes (pitch MW), `y*` y planes
// (pitch W) of fields 0 and 1.
template <typename T, class Pol, int DIM, int W, int MW>
__device__ __forceinline__ void compute_rhs(const StageArgs<T>& A, const Pol& pol, const T* mc, const T* mm,
                                            const T* mp, int moff, const T* y0c, const T* y0m, const T* y0p,
                                            const T* y1c, const T* y1m, const T* y1p, int yoff, T* k) {
    const T lapmu = Pol::MU ? tile_lap<T, DIM, MW>(A, mc, mm, mp, moff) : (T)0;
    const T lapy0 = Pol::LAP_Y0 ? tile_lap<T, DIM, W>(A, y0c, y0m, y0p, yoff) : (T)0;
    const T lapy1 = Pol::LAP_Y1 ? tile_lap<T, DIM, W>(A, y1c, y1m, y1p, yoff) : (T)0;
    pol.rhs(A, lapmu, y0c[yoff], lapy0, Pol::NF > 1 ? y1c[yoff] : (T)0, lapy1, k);
}

// Writes k or the final state for field f at flat index idx.
template <typename T, int MODE>
__device__ __forceinline__ void emit(const StageArgs<T>& A, int f, int idx, T k) {
    if (MODE == MODE_K) {
        A.out[f][idx] = k;
    } else if (MODE == MODE_EULER_FINAL || MODE == MODE_MULTISTEP) {
        if (A.ulo[f]) {
            twosum_update(__ldg(A.u[f] + idx), __ldg(A.ulo[f] + idx), rmul(A.dtf, k), &A.out[f][idx],
                          &A.outlo[f][idx]);
        } else {
            A.out[f][idx] = rfma(A.dtf, k, __ldg(A.u[f] + idx));
        }
    } else {
        // phi += dt6 * (((k1 + 2 k2) + 2 k3) + k4)
        T s = radd(__ldg(A.k1[f] + idx), rmul((T)2, __ldg(A.k2[f] + idx)));
        s = radd(s, rmul((T)2, __ldg(A.kin[f] + idx)));
        s = radd(s, k);
        if (A.ulo[f]) {
            twosum_update(__ldg(A.u[f] + idx), __ldg(A.ulo[f] + idx), rmul(A.dtf, s), &A.out[f][idx],
                          &A.outlo[f][idx]);
        } else {
            A.out[f][idx] = rfma(A.dtf, s, __ldg(A.u[f] + idx));
        }
    }
}

// Ghost cells of the new state: the reference leaves the BC-refreshed ghosts
// of the old state in place (BCs run at the start of the step and the updates
// add 0 there), i.e. the mapped value of the OLD state.
template <typename T, int DIM>
__device__ __forceinline__ void write_ghost(const StageArgs<T>& A, int nf, int px, int py, int pz) {
    int src;
    double cval;
    int dst = A.L.origin + px + A.L.s[1] * py + A.L.s[2] * pz;
    bool cst = map3<DIM>(A.L, px, py, pz, &src, &cval) == MAP_CONST;
    for (int f = 0; f < nf; ++f) {
        A.out[f][dst] = cst ? (T)cval : __ldg(A.u[f] + src);
        if (A.ulo[f]) A.outlo[f][dst] = cst ? (T)0 : __ldg(A.ulo[f] + src);
    }
}

// Ghost layers of the new state next to the TX x TY tile at (x0, y0): the
// final stage writes them so the new state's stored array is complete.
template <typename T, int DIM, int NF, int TX, int TY, int NT>
__device__ __forceinline__ void box_ghosts(const StageArgs<T>& A, int x0, int y0) {
    const int n0 = A.L.n[0], n1 = A.L.n[1], gl = A.L.ghost;
    // x faces
    if (x0 == 0 || x0 + TX >= n0) {
        for (int i = threadIdx.x; i < TY * gl; i += NT) {
            const int py = y0 + i / gl, l = 1 + i % gl;
            if (DIM >= 2 && py >= n1) continue;
            if (DIM < 2 && i / gl > 0) continue;
            if (x0 == 0) write_ghost<T, DIM>(A, NF, -l, DIM >= 2 ? py : 0, 0);
            if (x0 + TX >= n0) write_ghost<T, DIM>(A, NF, n0 - 1 + l, DIM >= 2 ? py : 0, 0);
        }
    }
    if (DIM >= 2 && (y0 == 0 || y0 + TY >= n1)) {
        for (int i = threadIdx.x; i < TX * gl; i += NT) {
            const int px = x0 + i % TX, l = 1 + i / TX;
            if (px >= n0) continue;
            if (y0 == 0) write_ghost<T, DIM>(A, NF, px, -l, 0);
            if (y0 + TY >= n1) write_ghost<T, DIM>(A, NF, px, n1 - 1 + l, 0);
        }
    }
}

// ---------------------------------------------------------------------------
// 1-D / 2-D: box tile
// ---------------------------------------------------------------------------
// Shared memory of one box tile.
template <typename T, class Pol, int DIM, int TX, int TY>
struct BoxSmem {
    using P = Pol;
    static constexpr int H = P::H, HY = DIM >= 2 ? P::H : 0;
    static constexpr int WX = TX + 2 * H, WY = TY + 2 * HY;
    static constexpr int MX = TX + 2, MY = TY + (DIM >= 2 ? 2 : 0);
    T ys[P::NF][WY * WX];
    T ms[P::MU ? MY * MX : 1];
};

// One TX x TY tile whose first physical cell is (x0, y0).
template <typename T, class Pol, int DIM, int MODE, int TX, int TY, int NT>
__device__ __forceinline__ void box_tile(const StageArgs<T>& A, const Pol& pol, BoxSmem<T, Pol, DIM, TX, TY>& sm,
                                         int x0, int y0) {
    using P = Pol;
    using S = BoxSmem<T, Pol, DIM, TX, TY>;
    constexpr int NF = P::NF, H = S::H, HY = S::HY, WX = S::WX, WY = S::WY, MX = S::MX, MY = S::MY;
    T(&ys)[NF][WY * WX] = sm.ys;
    T* ms = sm.ms;

    const int n0 = A.L.n[0], n1 = A.L.n[1];
    const bool interior = x0 - H >= 0 && x0 + TX + H <= n0 && (DIM < 2 || (y0 - HY >= 0 && y0 + TY + HY <= n1));

    // fixed trip counts: every load of a phase is issued before any is used
    constexpr int NLOAD = (WX * WY + NT - 1) / NT;
#pragma unroll
    for (int it = 0; it < NLOAD; ++it) {
        const int i = threadIdx.x + it * NT;
        if (i >= WX * WY) break;
        const int lx = i % WX, ly = i / WX;
        const int px = x0 - H + lx, py = y0 - HY + ly;
#pragma unroll
        for (int f = 0; f < NF; ++f) ys[f][i] = load_y<T, DIM>(A, f, px, py, 0, interior);
    }
    __syncthreads();

    if (P::MU) {
        constexpr int NMU = (MX * MY + NT - 1) / NT;
#pragma unroll
        for (int it = 0; it < NMU; ++it) {
            const int i = threadIdx.x + it * NT;
            if (i >= MX * MY) break;
            const int lx = i % MX, ly = i / MX;
            const int px = x0 - 1 + lx, py = y0 - (DIM >= 2 ? 1 : 0) + ly;
            int qx = px, qy = py;
            double cval = 0.0;
            bool cst = false;
            if (!interior) {
                cst = mu_axis(px, n0, A.L.bc[0], A.L.bc[1], A.L.bcv[0], A.L.bcv[1], &qx, &cval) == MAP_CONST;
                if (!cst && DIM >= 2)
                    cst = mu_axis(py, n1, A.L.bc[2], A.L.bc[3], A.L.bcv[2], A.L.bcv[3], &qy, &cval) == MAP_CONST;
            }
            T v;
            if (cst) {
                v = (T)cval;
            } else {
                const int off = (qx - x0 + H) + (qy - y0 + HY) * WX;
                v = compute_mu<T, Pol, DIM, WX>(A, pol, ys[0], nullptr, nullptr, ys[NF - 1], off);
            }
            ms[i] = v;
        }
        __syncthreads();
    }

    constexpr int NOUT = (TX * TY + NT - 1) / NT;
#pragma unroll
    for (int it = 0; it < NOUT; ++it) {
        const int i = threadIdx.x + it * NT;
        if (i >= TX * TY) break;
        const int lx = i % TX, ly = i / TX;
        const int px = x0 + lx, py = y0 + ly;
        if (px >= n0 || (DIM >= 2 && py >= n1)) continue;
        const int yoff = (lx + H) + (ly + HY) * WX;
        const int moff = (lx + 1) + (ly + (DIM >= 2 ? 1 : 0)) * MX;
        T k[2];
        compute_rhs<T, Pol, DIM, WX, MX>(A, pol, ms, nullptr, nullptr, moff, ys[0], nullptr, nullptr, ys[NF - 1],
                                         nullptr, nullptr, yoff, k);
        const int idx = A.L.origin + px + A.L.s[1] * py;
#pragma unroll
        for (int f = 0; f < NF; ++f) emit<T, MODE>(A, f, idx, k[f]);
        if (MODE == MODE_MULTISTEP) A.mu_out[idx] = ms[moff];
    }

    if (MODE == MODE_MULTISTEP && !interior) {
        // ghost layer 1 of mu: the BC-mapped ring values (the STEADY field is
        // zeroed, written, then its BCs run before the TRANSIENT step reads it)
        for (int i = threadIdx.x; i < MX * MY; i += NT) {
            const int lx = i % MX, ly = i / MX;
            const int px = x0 - 1 + lx, py = y0 - (DIM >= 2 ? 1 : 0) + ly;
            if (px < -1 || px > n0 || (DIM >= 2 && (py < -1 || py > n1))) continue;  // past ghost layer 1
            const bool outx = px < 0 || px >= n0, outy = DIM >= 2 && (py < 0 || py >= n1);
            if (outx == outy) continue;  // interior or corner
            if (outx && (py < y0 || py >= y0 + TY)) continue;  // owned by the neighbour tile row
            if (outy && (px < x0 || px >= x0 + TX)) continue;
            if (A.L.bc[(outx ? 0 : 2) + ((outx ? px : py) < 0 ? 0 : 1)] == PHIX_BC_NONE) continue;
            A.mu_out[A.L.origin + px + A.L.s[1] * py] = ms[i];
        }
    }

    if (MODE != MODE_K && !interior) box_ghosts<T, DIM, NF, TX, TY, NT>(A, x0, y0);
}

// Single field: one CTA per tile.
template <typename T, class Pol, int DIM, int MODE, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT) stage_box(const StageArgs<T> A, const Pol pol) {
    __shared__ BoxSmem<T, Pol, DIM, TX, TY> sm;
    box_tile<T, Pol, DIM, MODE, TX, TY, NT>(A, pol, sm, blockIdx.x * TX, blockIdx.y * TY);
}

// Many independent fields in one persistent launch: CTA b walks the tile list
// b, b + gridDim.x, ...; tile t = (instance, x0, y0) and the instance's stage
// arguments come from `args` (one StageArgs per instance for this stage).
struct BatchTile {
    int inst, x0, y0, pad;
};

template <typename T, class Pol, int MODE, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT) stage_box_batched(const StageArgs<T>* __restrict__ args,
                                                        const BatchTile* __restrict__ tiles, int ntiles,
                                                        const Pol pol) {
    __shared__ BoxSmem<T, Pol, 2, TX, TY> sm;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const BatchTile bt = tiles[t];
        box_tile<T, Pol, 2, MODE, TX, TY, NT>(args[bt.inst], pol, sm, bt.x0, bt.y0);
        __syncthreads();  // shared memory is reused by the next tile
    }
}

// ---------------------------------------------------------------------------
// 3-D: in-plane tile marching along z
// ---------------------------------------------------------------------------
template <typename T, class Pol, int TX, int TY>
struct March3D {
    static constexpr int NF = Pol::NF, H = Pol::H;
    static constexpr int WX = TX + 2 * H, WY = TY + 2 * H, WP = WX * WY;  // y plane
    static constexpr int MX = TX + 2, MY = TY + 2, MP = MX * MY;         // mu plane
    static constexpr int NYR = 5, NMR = 4;                               // ring depths
    static constexpr size_t smem_bytes() {
        return sizeof(T) * ((size_t)NF * NYR * WP + (Pol::MU ? (size_t)NMR * MP : 0));
    }
};

// The boundary mapping of one in-plane coordinate, resolved once per CTA:
// the mapped coordinate q, or (q == MAP_CONST_Q) the constant the mapping
// gives (map_axis / mu_axis semantics).
constexpr int MAP_CONST_Q = -0x40000000;

template <typename T, class Pol, int MODE, int TX, int TY, int RZ, int NT>
__global__ void __launch_bounds__(NT) stage_march3d(const StageArgs<T> A, const Pol pol) {
    using G = March3D<T, Pol, TX, TY>;
    constexpr int NF = G::NF, H = G::H, WX = G::WX, WY = G::WY, WP = G::WP, MX = G::MX, MY = G::MY, MP = G::MP;
    constexpr int NYR = G::NYR, NMR = G::NMR;
    constexpr bool MU = Pol::MU;
    constexpr int YC = (WP + NT - 1) / NT, MC = (MP + NT - 1) / NT, KC = (TX * TY + NT - 1) / NT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* ysb = reinterpret_cast<T*>(smem_raw);   // [NF][NYR][WP]
    T* msb = ysb + (size_t)NF * NYR * WP;      // [NMR][MP]
    // per-axis maps: y planes (global x, s1 * y) and mu planes (tile offsets)
    __shared__ int yqx[WX], yqy[WY], mqx[MX], mqy[MY];
    __shared__ double ycx[WX], ycy[WY], mcx[MX], mcy[MY];

    const Layout& L = A.L;
    const int n0 = L.n[0], n1 = L.n[1], n2 = L.n[2];
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * RZ;
    const int z1 = min(z0 + RZ, n2);

    for (int i = threadIdx.x; i < WX + WY + MX + MY; i += NT) {
        int q;
        double cv = 0.0;
        if (i < WX) {
            const bool c = map_axis(x0 - H + i, n0, L.bc[0], L.bc[1], L.bcv[0], L.bcv[1], L.ghost, &q, &cv) == MAP_CONST;
            yqx[i] = c ? MAP_CONST_Q : q;
            ycx[i] = cv;
        } else if (i < WX + WY) {
            const int k = i - WX;
            const bool c = map_axis(y0 - H + k, n1, L.bc[2], L.bc[3], L.bcv[2], L.bcv[3], L.ghost, &q, &cv) == MAP_CONST;
            yqy[k] = c ? MAP_CONST_Q : L.s[1] * q;
            ycy[k] = cv;
        } else if (i < WX + WY + MX) {
            const int k = i - WX - WY;
            const bool c = mu_axis(x0 - 1 + k, n0, L.bc[0], L.bc[1], L.bcv[0], L.bcv[1], &q, &cv) == MAP_CONST;
            mqx[k] = c ? MAP_CONST_Q : q - x0 + H;
            mcx[k] = cv;
        } else {
            const int k = i - WX - WY - MX;
            const bool c = mu_axis(y0 - 1 + k, n1, L.bc[2], L.bc[3], L.bcv[2], L.bcv[3], &q, &cv) == MAP_CONST;
            mqy[k] = c ? MAP_CONST_Q : (q - y0 + H) * WX;
            mcy[k] = cv;
        }
    }
    __syncthreads();

    auto yslot = [&](int f, int z) -> T* { return ysb + ((size_t)f * NYR + (unsigned)(z + 8 * NYR) % NYR) * WP; };
    auto mslot = [&](int z) -> T* { return msb + (size_t)((unsigned)(z + 8 * NMR) % NMR) * MP; };

    // plane z of the stage state y = u (+ a kin), tile + H: map3's order of
    // constants (x, then y, then z)
    auto form_y = [&](int z) {
        int qz;
        double zc = 0.0;
        const bool zcst = map_axis(z, n2, L.bc[4], L.bc[5], L.bcv[4], L.bcv[5], L.ghost, &qz, &zc) == MAP_CONST;
        const int zoff = L.origin + L.s[2] * qz;
        T* dst[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) dst[f] = yslot(f, z);
#pragma unroll
        for (int c = 0; c < YC; ++c) {
            const int i = threadIdx.x + c * NT;
            if (c + 1 < YC || i < WP) {
                const int lx = i % WX, ly = i / WX;
                const int qx = yqx[lx], qy = yqy[ly];
                const bool cst = qx == MAP_CONST_Q || qy == MAP_CONST_Q || zcst;
                const double cv = qx == MAP_CONST_Q ? ycx[lx] : qy == MAP_CONST_Q ? ycy[ly] : zc;
                const int idx = zoff + qx + qy;
#pragma unroll
                for (int f = 0; f < NF; ++f) {
                    T v;
                    if (cst) {
                        v = (T)cv;
                    } else {
                        v = __ldg(A.u[f] + idx);
                        if (A.kin[f] != nullptr) v = rfma(A.a, __ldg(A.kin[f] + idx), v);
                    }
                    dst[f][i] = v;
                }
            }
        }
    };
    // mu at plane z: mu_axis's order of constants (z, then x, then y)
    auto form_mu = [&](int z) {
        int qz = z;
        double zc = 0.0;
        const bool zcst = mu_axis(z, n2, L.bc[4], L.bc[5], L.bcv[4], L.bcv[5], &qz, &zc) == MAP_CONST;
        T* dst = mslot(z);
        const T* yc0 = yslot(0, qz);
        const T* ym0 = yslot(0, qz - 1);
        const T* yp0 = yslot(0, qz + 1);
        const T* yc1 = yslot(NF - 1, qz);
#pragma unroll
        for (int c = 0; c < MC; ++c) {
            const int i = threadIdx.x + c * NT;
            if (c + 1 < MC || i < MP) {
                const int lx = i % MX, ly = i / MX;
                const int ox = mqx[lx], oy = mqy[ly];
                T v;
                if (zcst) v = (T)zc;
                else if (ox == MAP_CONST_Q) v = (T)mcx[lx];
                else if (oy == MAP_CONST_Q) v = (T)mcy[ly];
                else v = compute_mu<T, Pol, 3, WX>(A, pol, yc0, ym0, yp0, yc1, ox + oy);
                dst[i] = v;
            }
        }
    };

    // prologue: y planes z0-2 .. z0+1 (z0-1 .. z0 for halo 1), mu planes z0-1, z0
    for (int z = z0 - H; z < z0 + H; ++z) form_y(z);
    __syncthreads();
    if (MU) {
        form_mu(z0 - 1);
        form_mu(z0);
    }

    for (int z = z0; z < z1; ++z) {
        form_y(z + H);
        __syncthreads();
        if (MU) {
            form_mu(z + 1);
            __syncthreads();
        }
        const T* y0c = yslot(0, z);
        const T* y0m = yslot(0, z - 1);
        const T* y0p = yslot(0, z + 1);
        const T* y1c = yslot(NF - 1, z);
        const T* y1m = yslot(NF - 1, z - 1);
        const T* y1p = yslot(NF - 1, z + 1);
        const T* mc = mslot(z);
        const T* mm = mslot(z - 1);
        const T* mp = mslot(z + 1);
        const int zidx = L.origin + L.s[2] * z;
#pragma unroll
        for (int c = 0; c < KC; ++c) {
            const int i = threadIdx.x + c * NT;
            if (c + 1 < KC || i < TX * TY) {
                const int lx = i % TX, ly = i / TX;
                const int px = x0 + lx, py = y0 + ly;
                if (px < n0 && py < n1) {
                    const int yoff = (lx + H) + (ly + H) * WX;
                    const int moff = (lx + 1) + (ly + 1) * MX;
                    T k[2];
                    compute_rhs<T, Pol, 3, WX, MX>(A, pol, mc, mm, mp, moff, y0c, y0m, y0p, y1c, y1m, y1p, yoff, k);
                    const int idx = zidx + px + L.s[1] * py;
#pragma unroll
                    for (int f = 0; f < NF; ++f) emit<T, MODE>(A, f, idx, k[f]);
                }
            }
        }
        if (MODE != MODE_K) {
            const bool in_xy = x0 - H >= 0 && x0 + TX + H <= n0 && y0 - H >= 0 && y0 + TY + H <= n1;
            const int gl = L.ghost;
            if (!in_xy) {
                if (x0 == 0 || x0 + TX >= n0)
                    for (int i = threadIdx.x; i < TY * gl; i += NT) {
                        const int py = y0 + i / gl, l = 1 + i % gl;
                        if (py >= n1) continue;
                        if (x0 == 0) write_ghost<T, 3>(A, NF, -l, py, z);
                        if (x0 + TX >= n0) write_ghost<T, 3>(A, NF, n0 - 1 + l, py, z);
                    }
                if (y0 == 0 || y0 + TY >= n1)
                    for (int i = threadIdx.x; i < TX * gl; i += NT) {
                        const int px = x0 + i % TX, l = 1 + i / TX;
                        if (px >= n0) continue;
                        if (y0 == 0) write_ghost<T, 3>(A, NF, px, -l, z);
                        if (y0 + TY >= n1) write_ghost<T, 3>(A, NF, px, n1 - 1 + l, z);
                    }
            }
            if (z == 0 || z == n2 - 1)
                for (int i = threadIdx.x; i < TX * TY * gl; i += NT) {
                    const int lx = i % TX, ly = (i / TX) % TY, l = 1 + i / (TX * TY);
                    const int px = x0 + lx, py = y0 + ly;
                    if (px >= n0 || py >= n1) continue;
                    if (z == 0) write_ghost<T, 3>(A, NF, px, py, -l);
                    if (z == n2 - 1) write_ghost<T, 3>(A, NF, px, py, n2 - 1 + l);
                }
        }
    }
}

}  // namespace phix
