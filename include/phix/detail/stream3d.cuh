// stream3d.cuh -- one RK4 / Euler stage of the chemical-potential physics (CH,
// coupled CH+AC) on 3-D grids, streamed through z with the z-neighbours in
// registers and the input planes staged by TMA.
//
// Each CTA owns a TX x TY in-plane tile and marches a range of z planes; each
// of its (TX + 4) x (TY + 4) threads owns one (x, y) column of the tile + 2.
// Per input plane p:
//   * the planes of u (and of the previous stage's k) arrive by TMA
//     (cp.async.bulk.tensor.3d, one box per array and field) into a ring of
//     slots, one mbarrier per slot, two (FP64) or three (FP32) planes ahead
//     of their use; one thread waits for each copy, the others at the CTA
//     barrier;
//   * every thread forms its column's stage state y = u + a k_prev
//     (kernel_rk4_tmp, Solver.cu:49-56), keeps it in a register window along z
//     and writes it into a shared plane (in-plane neighbours only);
//   * threads of the tile + 1 form mu at plane p-1 (makeStencilOnExprTerm,
//     Equation.cu:537-594), kept in a register window and one shared plane;
//   * threads of the tile form the right-hand side at plane p-2 (every DSL
//     term, Equation.cu:257-276) and write k, or the new state
//     (kernel_rk4_update / kernel_axpy, Solver.cu:30-71).
// The z-neighbours of every stencil come from registers, the in-plane ones from
// shared memory, and each thread's offsets are fixed for the whole march, so a
// stage costs a few shared-memory accesses per cell and no index arithmetic.
//
// Boundaries: z periodic (the plane index wraps before the copy); x and y
// periodic or zero-flux.  Input cells outside the grid are replaced after the
// copy by their BC-mapped values (map3, the ghost fill's values); mu outside
// the grid on a zero-flux side is computed at the clamped cell (mu_axis), on a
// periodic side at the image.  Every value sees the operations of
// stage_march3d in the same order (the Laplacian of tile_lap, the policy's mu
// and rhs, emit), so the bits equal that kernel's.
#pragma once

#include <cuda.h>
#include <stdint.h>

#include "phix/detail/march3d_fused.cuh"
#include "phix/detail/stage.cuh"

namespace phix {

template <typename T>
struct Stream3Args {
    StageArgs<T> S;
    CUtensorMap tu[2];  // u of each field
    CUtensorMap tk[2];  // the previous stage's k of each field (when S.kin is set)
    int rz;             // output planes per CTA
    int* err;           // set when a plane copy did not arrive in time
};

template <typename T, class Pol, int TX, int TY, bool FINAL>
struct Stream3 {
    static constexpr int NF = Pol::NF, H = Pol::H;
    static constexpr int NX = TX + 2 * H, NY = TY + 2 * H, NT = NX * NY;  // one thread per column of the tile + 2
    static constexpr int VEC = 16 / (int)sizeof(T);
    static constexpr int WB = (NX + VEC - 1 + VEC - 1) / VEC * VEC;  // box width = plane pitch (16-byte rows)
    static constexpr int HB = NY;
    static constexpr int PL = (WB * HB * (int)sizeof(T) + 127) / 128 * 128 / (int)sizeof(T);  // 128-byte slots
    // input slots: LA planes in flight beyond the plane in use; the final
    // stage keeps planes p-2 .. p resident (it reads u and the previous k of
    // plane p-2 from them), the others only plane p
    static constexpr int RES = FINAL ? 3 : 1;
    static constexpr int LA = FINAL ? (sizeof(T) == 4 ? 3 : 2) : (sizeof(T) == 4 ? 6 : 4), NS = RES + LA;
    static constexpr int NY_R = 4, NM_R = 2;  // shared planes of y (p-3 .. p) and mu (p-2, p-1)
    static constexpr size_t OFF_IN = 0;                                        // [NS][2 arrays][NF][PL]
    static constexpr size_t OFF_Y = OFF_IN + (size_t)NS * 2 * NF * PL;          // [NY_R][NF][PL]
    static constexpr size_t OFF_M = OFF_Y + (size_t)NY_R * NF * PL;            // [NM_R][PL]
    static constexpr size_t ELEMS = OFF_M + (size_t)NM_R * PL;
    static constexpr size_t BAR_OFF = (ELEMS * sizeof(T) + 7) / 8 * 8;
    static constexpr size_t smem_bytes() { return 128 + BAR_OFF + NS * 8; }
    static constexpr uint32_t BOX_BYTES = (uint32_t)(WB * HB * sizeof(T));
    static_assert(Pol::MU && H == 2, "the streaming 3-D stage is built for the chemical-potential physics");
    static_assert(WB <= 256 && HB <= 256 && NT <= 1024, "tile too large");
};

template <typename T, class Pol, int MODE, int TX, int TY>
__global__ void __launch_bounds__(Stream3<T, Pol, TX, TY, MODE != MODE_K>::NT)
    stage_stream3d(const __grid_constant__ Stream3Args<T> A) {
    using G = Stream3<T, Pol, TX, TY, MODE != MODE_K>;
    constexpr int NF = G::NF, H = G::H, NX = G::NX, WB = G::WB, PL = G::PL, NS = G::NS;
    constexpr int NYR = G::NY_R, NMR = G::NM_R;
    const Pol pol{};
    const StageArgs<T>& S = A.S;
    const Layout& L = S.L;
    extern __shared__ unsigned char s3_raw[];
    T* sm = reinterpret_cast<T*>((reinterpret_cast<uintptr_t>(s3_raw) + 127) & ~(uintptr_t)127);
    uint64_t* bars = reinterpret_cast<uint64_t*>(reinterpret_cast<unsigned char*>(sm) + G::BAR_OFF);

    const int n0 = L.n[0], n1 = L.n[1], n2 = L.n[2], gh = L.ghost;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int z0 = blockIdx.z * A.rz, z1 = min(z0 + A.rz, n2);
    const bool has_k = S.kin[0] != nullptr;
    const int sh = ((gh - H) % G::VEC + G::VEC) % G::VEC;  // boxes start on 16-byte boundaries
    const bool inner = x0 - H >= 0 && x0 + TX + H <= n0 && y0 - H >= 0 && y0 + TY + H <= n1;

    // this thread's column
    const int cx = threadIdx.x % NX, cy = threadIdx.x / NX;
    const int lx = cx - H, ly = cy - H, px = x0 + lx, py = y0 + ly;
    const int po = (cx + sh) + cy * WB;  // its cell in every plane slot
    const bool in_r1 = lx >= -1 && lx <= TX && ly >= -1 && ly <= TY;
    const bool in_tile = lx >= 0 && lx < TX && ly >= 0 && ly < TY && px < n0 && py < n1;
    const bool ood = px < 0 || px >= n0 || py < 0 || py >= n1;
    // mu of a cell outside the grid on a zero-flux side is the clamped cell's
    int mx = lx, my = ly;
    if (px < 0 && L.bc[0] == PHIX_BC_NOFLUX) mx = -x0;
    if (px >= n0 && L.bc[1] == PHIX_BC_NOFLUX) mx = n0 - 1 - x0;
    if (py < 0 && L.bc[2] == PHIX_BC_NOFLUX) my = -y0;
    if (py >= n1 && L.bc[3] == PHIX_BC_NOFLUX) my = n1 - 1 - y0;
    const int pm = (mx + H + sh) + (my + H) * WB;  // in-plane stencil centre of this thread's mu
    // in-plane part of the BC-mapped stored index of this column (periodic / zero-flux: never constant)
    int gxy = 0;
    if (ood) {
        int qx, qy;
        double cval;
        map_axis(px, n0, L.bc[0], L.bc[1], L.bcv[0], L.bcv[1], gh, &qx, &cval);
        map_axis(py, n1, L.bc[2], L.bc[3], L.bcv[2], L.bcv[3], gh, &qy, &cval);
        gxy = qx + L.s[1] * qy;
    }
    const int gtile = px + L.s[1] * py;  // stored offset of a tile cell (z excluded)

    auto zwrap = [&](int z) { const int r = z % n2; return r < 0 ? r + n2 : r; };
    auto in_slot = [&](int arr, int f, int z) -> T* {
        return sm + G::OFF_IN + ((size_t)(((unsigned)(z + 8 * NS) % NS) * 2 + arr) * NF + f) * PL;
    };
    auto y_slot = [&](int f, int z) -> T* { return sm + G::OFF_Y + ((size_t)((unsigned)(z + 8 * NYR) % NYR) * NF + f) * PL; };
    auto m_slot = [&](int z) -> T* { return sm + G::OFF_M + (size_t)((unsigned)(z + 8 * NMR) % NMR) * PL; };
    auto bar = [&](int z) -> uint64_t* { return bars + (unsigned)(z + 8 * NS) % NS; };

    const int t_first = z0 - H, t_last = z1 + H - 1;  // input planes
    auto issue = [&](int t) {  // thread 0
        uint64_t* b = bar(t);
        m2::arrive_expect_tx(b, G::BOX_BYTES * NF * (has_k ? 2 : 1));
        const int xs = x0 - H + gh - sh, ys = y0 - H + gh, zs = zwrap(t) + gh;
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            m2::tma_box3(in_slot(0, f, t), &A.tu[f], xs, ys, zs, b);
            if (has_k) m2::tma_box3(in_slot(1, f, t), &A.tk[f], xs, ys, zs, b);
        }
    };
    if (threadIdx.x == 0) {
        for (int i = 0; i < NS; ++i) m2::bar_init(bars + i, 1);
        m2::fence_bar_init();
    }
    __syncthreads();
    constexpr int LA = G::LA;
    if (threadIdx.x == 0)
        for (int t = t_first; t < t_first + LA && t <= t_last; ++t) issue(t);

    // register windows along z: c at p-2 .. p, eta at p-3 .. p, mu at p-3 .. p-1
    T w0[3], w1[4], wm[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) w0[i] = wm[i] = (T)0;
#pragma unroll
    for (int i = 0; i < 4; ++i) w1[i] = (T)0;
    const T a = S.a, i2x = S.i2[0], i2y = S.i2[1], i2z = S.i2[2];
    bool failed = false;
    int issued = min(t_first + LA - 1, t_last);  // last plane whose copy was issued
    constexpr bool FINAL = MODE == MODE_RK4_FINAL || MODE == MODE_EULER_FINAL;

    for (int p = t_first; p <= t_last; ++p) {
        // the final stage's k1, k2 and low parts of this thread's tile cell at
        // plane p-2, fetched now so that they arrive while the plane is formed
        T pk1[2] = {(T)0, (T)0}, pk2[2] = {(T)0, (T)0}, plo[2] = {(T)0, (T)0};
        if (FINAL && in_tile && p - 2 >= z0 && p - 2 < z1) {
            const int idx = L.origin + gtile + L.s[2] * (p - 2);
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                if (MODE == MODE_RK4_FINAL) {
                    pk1[f] = __ldg(S.k1[f] + idx);
                    pk2[f] = __ldg(S.k2[f] + idx);
                }
                if (S.ulo[f]) plo[f] = __ldg(S.ulo[f] + idx);
            }
        }
        // ---- the input plane p: one thread waits for its copy, the others at
        //      the CTA barrier; then BC-map this column if it lies outside the grid
        bool ok = true;
        if (threadIdx.x == 0) ok = m2::bar_wait_sleep(bar(p), (uint32_t)(((p - t_first) / NS) & 1), m2::WAIT_NS);
        if (__syncthreads_or(!ok)) { failed = true; break; }
        T y[2];
        if (!ood) {
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                const T u = in_slot(0, f, p)[po];
                y[f] = has_k ? rfma(a, in_slot(1, f, p)[po], u) : u;
            }
        } else {
            const int idx = L.origin + gxy + L.s[2] * zwrap(p);
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                const T u = __ldg(S.u[f] + idx);
                y[f] = has_k ? rfma(a, __ldg(S.kin[f] + idx), u) : u;
            }
        }
        w0[0] = w0[1]; w0[1] = w0[2]; w0[2] = y[0];
        if (NF > 1) { w1[0] = w1[1]; w1[1] = w1[2]; w1[2] = w1[3]; w1[3] = y[NF - 1]; }
#pragma unroll
        for (int f = 0; f < NF; ++f) y_slot(f, p)[po] = y[f];
        __syncthreads();
        // the slot of plane p - RES is free (last read by step p-1): plane p + LA into it
        if (threadIdx.x == 0 && p + LA <= t_last) {
            m2::fence_proxy_async();
            issue(p + LA);
            issued = p + LA;
        }
        // ---- mu at plane p-1 on the tile + 1
        if (p - 1 >= z0 - 1 && p - 1 <= z1) {
            if (in_r1) {
                const T* c = y_slot(0, p - 1);
                const T cc = w0[1];
                const T v2 = rmul((T)2, cc);
                const T tx = second_diff(c[pm + 1], v2, c[pm - 1]);
                const T ty = second_diff(c[pm + WB], v2, c[pm - WB]);
                const T tz = second_diff(w0[2], v2, w0[0]);
                const T lap = lap_combine<T, 3>(tx, ty, tz, i2x, i2y, i2z);
                const T mu = pol.mu(S, cc, lap, NF > 1 ? w1[2] : (T)0);
                wm[0] = wm[1]; wm[1] = wm[2]; wm[2] = mu;
                m_slot(p - 1)[po] = mu;
            }
        }
        __syncthreads();
        // ---- the right-hand side at plane p-2 on the tile
        const int z = p - 2;
        if (z >= z0 && z < z1) {
            if (in_tile) {
                const T* m = m_slot(z);
                const T mv2 = rmul((T)2, wm[1]);
                const T mtx = second_diff(m[po + 1], mv2, m[po - 1]);
                const T mty = second_diff(m[po + WB], mv2, m[po - WB]);
                const T mtz = second_diff(wm[2], mv2, wm[0]);
                const T lapmu = lap_combine<T, 3>(mtx, mty, mtz, i2x, i2y, i2z);
                T lapy1 = (T)0;
                if (Pol::LAP_Y1) {
                    const T* e = y_slot(NF - 1, z);
                    const T ev2 = rmul((T)2, w1[1]);
                    const T etx = second_diff(e[po + 1], ev2, e[po - 1]);
                    const T ety = second_diff(e[po + WB], ev2, e[po - WB]);
                    const T etz = second_diff(w1[2], ev2, w1[0]);
                    lapy1 = lap_combine<T, 3>(etx, ety, etz, i2x, i2y, i2z);
                }
                T k[2];
                pol.rhs(S, lapmu, w0[0], (T)0, NF > 1 ? w1[1] : (T)0, lapy1, k);
                const int idx = L.origin + gtile + L.s[2] * z;
#pragma unroll
                for (int f = 0; f < NF; ++f) {
                    if constexpr (MODE == MODE_K) {
                        S.out[f][idx] = k[f];
                    } else {
                        // emit's arithmetic, with u (and k3) from the plane's input slot
                        const T u = in_slot(0, f, z)[po];
                        T d;
                        if constexpr (MODE == MODE_RK4_FINAL) {
                            // phi += dt6 * (((k1 + 2 k2) + 2 k3) + k4)
                            T sum = radd(pk1[f], rmul((T)2, pk2[f]));
                            sum = radd(sum, rmul((T)2, in_slot(1, f, z)[po]));
                            d = radd(sum, k[f]);
                        } else {
                            d = k[f];
                        }
                        if (S.ulo[f]) twosum_update(u, plo[f], rmul(S.dtf, d), &S.out[f][idx], &S.outlo[f][idx]);
                        else S.out[f][idx] = rfma(S.dtf, d, u);
                    }
                }
            }
            if (MODE != MODE_K) {
                // ghost cells of the new state (the BC-mapped old state), as stage_march3d writes them
                if (!inner) {
                    if (x0 == 0 || x0 + TX >= n0)
                        for (int i = threadIdx.x; i < TY * gh; i += G::NT) {
                            const int qy = y0 + i / gh, l = 1 + i % gh;
                            if (qy >= n1) continue;
                            if (x0 == 0) write_ghost<T, 3>(S, NF, -l, qy, z);
                            if (x0 + TX >= n0) write_ghost<T, 3>(S, NF, n0 - 1 + l, qy, z);
                        }
                    if (y0 == 0 || y0 + TY >= n1)
                        for (int i = threadIdx.x; i < TX * gh; i += G::NT) {
                            const int qx = x0 + i % TX, l = 1 + i / TX;
                            if (qx >= n0) continue;
                            if (y0 == 0) write_ghost<T, 3>(S, NF, qx, -l, z);
                            if (y0 + TY >= n1) write_ghost<T, 3>(S, NF, qx, n1 - 1 + l, z);
                        }
                }
                if (z == 0 || z == n2 - 1)
                    for (int i = threadIdx.x; i < TX * TY * gh; i += G::NT) {
                        const int qx = x0 + i % TX, qy = y0 + (i / TX) % TY, l = 1 + i / (TX * TY);
                        if (qx >= n0 || qy >= n1) continue;
                        if (z == 0) write_ghost<T, 3>(S, NF, qx, qy, -l);
                        if (z == n2 - 1) write_ghost<T, 3>(S, NF, qx, qy, n2 - 1 + l);
                    }
            }
        }
        // slots written at step p + 1 (y of p + 1, mu of p) were last read
        // before one of the two barriers above
    }

    if (failed) {
        // a copy did not arrive in time: record it, and let the copies still in
        // flight land (bounded) before the CTA's shared memory is released
        if (threadIdx.x == 0) {
            atomicExch(A.err, 1);
            for (int t = issued - NS + 1; t <= issued; ++t)
                if (t >= t_first) m2::bar_wait(bar(t), (uint32_t)(((t - t_first) / NS) & 1), m2::WAIT_NS);
        }
        __syncthreads();
    }
}

}  // namespace phix
