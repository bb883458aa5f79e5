// stream3d.cuh -- one RK4 / Euler stage of the chemical-potential physics (CH,
// coupled CH+AC) on 3-D grids, streamed through z with the z-neighbours in
// registers and the input planes staged by TMA.
//
// Each CTA owns a TX x TY in-plane tile and marches a range of z planes.  Its
// threads cover the tile + 2: thread (cx, g) owns column cx and the R rows
// g R .. g R + R - 1 of it.  Per input plane p:
//   * the planes of u (and of the previous stage's k) arrive by TMA
//     (cp.async.bulk.tensor.3d, one box per array and field) into a ring of
//     slots, one mbarrier per slot, LA planes ahead of their use; every thread
//     waits for the copy it reads (suspended in the mbarrier's try_wait);
//   * every thread forms the stage state y = u + a k_prev of its R cells
//     (kernel_rk4_tmp, Solver.cu:49-56), keeps them in register windows along
//     z and writes them into a shared plane;
//   * cells of the tile + 1 form mu at plane p-1 (makeStencilOnExprTerm,
//     Equation.cu:537-594), kept in register windows and one shared plane;
//   * cells of the tile form the right-hand side at plane p-2 (every DSL term,
//     Equation.cu:257-276) and write k, or the new state (kernel_rk4_update /
//     kernel_axpy, Solver.cu:30-71).
// The z-neighbours of every stencil come from registers, so do the y-neighbours
// of a thread's inner rows; x-neighbours (and the y-neighbours of its first and
// last row) come from the shared planes.  The slot offsets are fixed for the
// whole march, so a stage costs a few shared-memory accesses per cell.  One CTA
// barrier per plane (after the stage-state store) orders every shared slot's
// reuse.  The k stages march four planes per pass, so that the ring positions
// of the windows and slots are compile-time; the update, whose extra operands
// leave no registers for that, rolls one plane at a time.
//
// Boundaries: z periodic (the plane index wraps before the copy); x and y
// periodic or zero-flux.  Input cells outside the grid are replaced after the
// copy by their BC-mapped values (map3, the ghost fill's values); mu outside
// the grid on a zero-flux side is computed at the clamped cell (mu_axis), on a
// periodic side at the image.  CTAs whose tile + 2 lies inside the grid take
// none of these paths.  Every value sees the operations of stage_march3d in the
// same order (the Laplacian of tile_lap, the policy's mu and rhs, emit), so the
// bits equal that kernel's.
#pragma once

#include <cuda.h>
#include <stdint.h>

#include <type_traits>

#include "phix/detail/march3d_fused.cuh"
#include "phix/detail/stage.cuh"

namespace phix {

template <typename T>
struct Stream3Args {
    StageArgs<T> S;
    CUtensorMap tu[2];  // u of each field
    CUtensorMap tk[2];  // the previous stage's k of each field (when S.kin is set)
    // final stages: k1, k2 and the low parts of each field, boxes of the tile
    // rows (TX + 16 bytes wide) that FP64 updates prefetch into L2 LA planes
    // ahead of their loads (FP32 updates measured faster without); bit 2 j + f
    // of pfm marks tq[j][f] as encoded
    CUtensorMap tq[3][2];
    int pfm;
    int rz;             // output planes per CTA
    int* err;           // set when a plane copy did not arrive in time
};

template <typename T, class Pol, int TX, int TY, int R, bool FINAL>
struct Stream3 {
    static constexpr int NF = Pol::NF, H = Pol::H;
    static constexpr int NX = TX + 2 * H, NY = TY + 2 * H;  // the tile + 2
    static constexpr int NG = NY / R, NT = NX * NG;          // one thread per column and group of R rows
    static constexpr int VEC = 16 / (int)sizeof(T);
    static constexpr int WB = (NX + VEC - 1 + VEC - 1) / VEC * VEC;  // box width = plane pitch (16-byte rows)
    static constexpr int HB = NY;
    static constexpr int PL = (WB * HB * (int)sizeof(T) + 127) / 128 * 128 / (int)sizeof(T);  // 128-byte slots
    // input slots: LA planes in flight beyond the plane in use; the final
    // stage keeps planes p-2 .. p resident (it reads u and the previous k of
    // plane p-2 from them), the others only plane p
    static constexpr int RES = FINAL ? 3 : 1;
    // one row per thread leaves room for a deeper ring; R rows per thread hold
    // R times the cells of a thread in every slot
    // (FP64 k stages on tiles of fewer than 8 rows: 2, so that three CTAs fit)
    static constexpr int LA = R > 1 ? 2 : FINAL ? (sizeof(T) == 4 ? 3 : 2) : (sizeof(T) == 4 ? 6 : TY < 8 ? 2 : 4);
    static constexpr int NS = RES + LA;
    // shared planes of y (p-3 .. p) and mu (p-2, p-1).  One CTA barrier per
    // plane (after the y store): every slot is rewritten only after the barrier
    // that follows its last read (y of p-4 was last read by the right-hand side
    // of p-2, mu of p-3 by that of p-1, input plane p-RES by step p-1)
    static constexpr int NY_R = 4, NM_R = 2;
    static constexpr size_t OFF_IN = 0;                               // [NS][2 arrays][NF][PL]
    static constexpr size_t OFF_Y = OFF_IN + (size_t)NS * 2 * NF * PL;  // [NY_R][NF][PL]
    static constexpr size_t OFF_M = OFF_Y + (size_t)NY_R * NF * PL;    // [NM_R][PL]
    // every row of a thread is computed, its stores masked: the stencils of the
    // outermost rows read one row beyond the last mu slot, into this padding
    static constexpr size_t ELEMS = OFF_M + (size_t)NM_R * PL + WB + 8;
    static constexpr size_t BAR_OFF = (ELEMS * sizeof(T) + 7) / 8 * 8;
    static constexpr size_t smem_bytes() { return 128 + BAR_OFF + NS * 8; }
    static constexpr uint32_t BOX_BYTES = (uint32_t)(WB * HB * sizeof(T));
    // CTAs per SM the registers are budgeted for: as many as the shared memory
    // holds with one row per thread (FP32 k stages and FP64 ones on tiles of
    // fewer than 8 rows: 3, else 2)
    static constexpr int MIN_CTAS = R == 1 ? ((sizeof(T) == 4 || TY < 8) && !FINAL ? 3 : 2) : 1;
    static_assert(Pol::MU && H == 2, "the streaming 3-D stage is built for the chemical-potential physics");
    static_assert(NY % R == 0 && R >= 1 && R <= 8, "the rows of the tile + 2 split into whole groups of R");
    static_assert(WB <= 256 && HB <= 256 && NT <= 1024, "tile too large");
};

template <typename T, class Pol, int MODE, int TX, int TY, int R>
__global__ void __launch_bounds__(Stream3<T, Pol, TX, TY, R, MODE != MODE_K>::NT,
                                  Stream3<T, Pol, TX, TY, R, MODE != MODE_K>::MIN_CTAS)
    stage_stream3d(const __grid_constant__ Stream3Args<T> A) {
    using G = Stream3<T, Pol, TX, TY, R, MODE != MODE_K>;
    constexpr int NF = G::NF, H = G::H, NX = G::NX, WB = G::WB, PL = G::PL, NS = G::NS, LA = G::LA;
    constexpr bool FINAL = MODE == MODE_RK4_FINAL || MODE == MODE_EULER_FINAL;
    const Pol pol{};
    const StageArgs<T>& S = A.S;
    const Layout& L = S.L;
    // 128-byte aligned slots; the offset is added to the shared array itself (not
    // through an integer) so that every slot access stays a shared-memory access
    extern __shared__ __align__(128) unsigned char s3_raw[];
    T* sm = reinterpret_cast<T*>(s3_raw + ((128u - (m2::saddr(s3_raw) & 127u)) & 127u));
    uint64_t* bars = reinterpret_cast<uint64_t*>(reinterpret_cast<unsigned char*>(sm) + G::BAR_OFF);

    const int n0 = L.n[0], n1 = L.n[1], n2 = L.n[2], gh = L.ghost;
    const int s1 = L.s[1], s2 = L.s[2];
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int z0 = blockIdx.z * A.rz, z1 = min(z0 + A.rz, n2);
    const bool has_k = S.kin[0] != nullptr;
    const int sh = ((gh - H) % G::VEC + G::VEC) % G::VEC;  // boxes start on 16-byte boundaries
    // the tile + 2 lies inside the grid: no BC mapping, no clamped mu
    const bool inner = x0 - H >= 0 && x0 + TX + H <= n0 && y0 - H >= 0 && y0 + TY + H <= n1;

    // this thread's column and rows: warps take 32 columns of one row group
    // (one bank each in a shared plane, no conflicts), the last threads the
    // NX - 32 columns left over in every group
    int cx, grp;
    if constexpr (NX > 32) {
        constexpr int MAIN = 32 * G::NG;
        if ((int)threadIdx.x < MAIN) {
            cx = threadIdx.x % 32;
            grp = threadIdx.x / 32;
        } else {
            cx = 32 + ((int)threadIdx.x - MAIN) % (NX - 32);
            grp = ((int)threadIdx.x - MAIN) / (NX - 32);
        }
    } else {
        cx = threadIdx.x % NX;
        grp = threadIdx.x / NX;
    }
    const int lx = cx - H, px = x0 + lx;
    const int ly0 = grp * R - H, py0 = y0 + ly0;  // its first row
    const int po = (cx + sh) + grp * R * WB;      // slot offset of its first row
    unsigned r1m = 0, tm = 0, oodm = 0;           // its rows on the tile + 1, on the tile, outside the grid
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int ly = ly0 + r, py = py0 + r;
        if (lx >= -1 && lx <= TX && ly >= -1 && ly <= TY) r1m |= 1u << r;
        if (lx >= 0 && lx < TX && ly >= 0 && ly < TY && px < n0 && py < n1) tm |= 1u << r;
        if (px < 0 || px >= n0 || py < 0 || py >= n1) oodm |= 1u << r;
    }
    // mu of a cell outside the grid on a zero-flux side is the clamped cell's:
    // the column shift (the rows' shifts are formed in the edge path)
    int mx = lx;
    if (px < 0 && L.bc[0] == PHIX_BC_NOFLUX) mx = -x0;
    if (px >= n0 && L.bc[1] == PHIX_BC_NOFLUX) mx = n0 - 1 - x0;
    const int pmx = mx - lx;
    // BC-mapped stored column (periodic / zero-flux: never a constant)
    int qx = px;
    if (oodm) {
        double cval;
        map_axis(px, n0, L.bc[0], L.bc[1], L.bcv[0], L.bcv[1], gh, &qx, &cval);
    }
    const int gtile = px + s1 * py0;  // stored offset of the first row (z excluded)

    auto zwrap = [&](int z) {
        if ((unsigned)z < (unsigned)n2) return z;
        const int r = z % n2;
        return r < 0 ? r + n2 : r;
    };
    // ring positions count from the first input plane t_first
    const int t_first = z0 - H, t_last = z1 + H - 1;
    auto in_base = [&](int slot) -> T* { return sm + G::OFF_IN + (size_t)slot * 2 * NF * PL; };
    auto issue = [&](int t, int slot) {  // thread 0
        uint64_t* b = bars + slot;
        m2::arrive_expect_tx(b, G::BOX_BYTES * NF * (has_k ? 2 : 1));
        const int xs = x0 - H + gh - sh, ys = y0 - H + gh, zs = zwrap(t) + gh;
        T* dst = in_base(slot);
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            m2::tma_box3(dst + f * PL, &A.tu[f], xs, ys, zs, b);
            if (has_k) m2::tma_box3(dst + (NF + f) * PL, &A.tk[f], xs, ys, zs, b);
        }
    };
    if (threadIdx.x == 0) {
        for (int i = 0; i < NS; ++i) m2::bar_init(bars + i, 1);
        m2::fence_bar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int t = t_first; t < t_first + LA && t <= t_last; ++t) issue(t, t - t_first);

    // register windows along z, per row, as rings over the plane's position
    // J = (p - t_first) mod 4, which the march below makes a compile-time
    // index: c of planes p-2 .. p, eta of p-3 .. p, mu of p-3 .. p-1
    T w0[R][4], w1[R][4], wm[R][4];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
        for (int i = 0; i < 4; ++i) w0[r][i] = w1[r][i] = wm[r][i] = (T)0;
    const T a = S.a, i2x = S.i2[0], i2y = S.i2[1], i2z = S.i2[2];
    bool failed = false;
    int issued = min(t_first + LA - 1, t_last);  // last plane whose copy was issued
    int si = 0;        // input slot of plane p
    uint32_t ph = 0;   // phase parity of the input slot's mbarrier

    // One input plane p.  Jc = 0..3: the plane's ring position (p - t_first)
    // mod 4, compile-time, which indexes the y and mu slots and the register
    // windows; Jc = -1: a rolling loop, the windows shifted by one plane and the
    // slots indexed at run time (the update's form: unrolled, its extra
    // operands exceed the register budget).  DO_MU: mu of plane p-1 is formed,
    // DO_K: the right-hand side of plane p-2.  False: a copy did not arrive.
    auto plane = [&](auto Jc, auto MUc, auto Kc, const int p) -> bool {
        constexpr bool SHIFT = decltype(Jc)::value < 0;
        constexpr int J = SHIFT ? 3 : decltype(Jc)::value;                   // window index of plane p
        constexpr int J1 = (J + 3) & 3, J2 = (J + 2) & 3, J3 = (J + 1) & 3;  // planes p-1, p-2, p-3
        constexpr bool DO_MU = decltype(MUc)::value, DO_K = decltype(Kc)::value;
        const int jy = SHIFT ? ((p - t_first) & 3) : J;  // y slot of plane p
        T* const in_p = in_base(si);
        T* const in_p2 = in_base(si >= 2 ? si - 2 : si + NS - 2);  // plane p-2 (final stage)
        T* const y_p = sm + G::OFF_Y + (size_t)jy * NF * PL;
        T* const y_p1 = sm + G::OFF_Y + (size_t)((jy + 3) & 3) * NF * PL;
        T* const y_p2 = sm + G::OFF_Y + (size_t)((jy + 2) & 3) * NF * PL;
        T* const m_p1 = sm + G::OFF_M + (size_t)((jy + 3) & 1) * PL;  // mu of plane p-1
        T* const m_p2 = sm + G::OFF_M + (size_t)((jy + 2) & 1) * PL;  // mu of plane p-2
        const int z = p - 2;
        if constexpr (SHIFT) {
            // planes p-2 .. p-1 (c), p-3 .. p-1 (eta) and p-3 .. p-2 (mu) move
            // to the window indices 1..2, 0..2 and 0..1
#pragma unroll
            for (int r = 0; r < R; ++r) {
                w0[r][1] = w0[r][2]; w0[r][2] = w0[r][3];
                w1[r][0] = w1[r][1]; w1[r][1] = w1[r][2]; w1[r][2] = w1[r][3];
                wm[r][0] = wm[r][1]; wm[r][1] = wm[r][2];
            }
        }

        // the final stage's k1, k2 and low parts of this thread's tile cells at
        // plane p-2, fetched now so that they arrive while the plane is formed
        T pk1[R][2], pk2[R][2], plo[R][2];
        if (FINAL && DO_K) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (!((tm >> r) & 1u)) continue;
                const int idx = L.origin + gtile + s1 * r + s2 * z;
#pragma unroll
                for (int f = 0; f < NF; ++f) {
                    if (MODE == MODE_RK4_FINAL) {
                        pk1[r][f] = __ldg(S.k1[f] + idx);
                        pk2[r][f] = __ldg(S.k2[f] + idx);
                    }
                    plo[r][f] = S.ulo[f] ? __ldg(S.ulo[f] + idx) : (T)0;
                }
            }
        }
        // ---- the input plane p: every thread waits for its copy (suspended in
        //      the mbarrier's try_wait, not spinning); cells outside the grid take
        //      their BC-mapped values.  A copy that does not land in time is
        //      agreed on at the barrier below.
        const bool ok = m2::bar_wait_sleep(bars + si, ph, m2::WAIT_NS);
        T y[R][2];
        if (!oodm) {
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int f = 0; f < NF; ++f) {
                    const T u = in_p[f * PL + po + r * WB];
                    y[r][f] = has_k ? rfma(a, in_p[(NF + f) * PL + po + r * WB], u) : u;
                }
        } else {
            const int zi = zwrap(p);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if ((oodm >> r) & 1u) {
                    int qy;
                    double cval;
                    map_axis(py0 + r, n1, L.bc[2], L.bc[3], L.bcv[2], L.bcv[3], gh, &qy, &cval);
                    const int idx = L.origin + qx + s1 * qy + s2 * zi;
#pragma unroll
                    for (int f = 0; f < NF; ++f) {
                        const T u = __ldg(S.u[f] + idx);
                        y[r][f] = has_k ? rfma(a, __ldg(S.kin[f] + idx), u) : u;
                    }
                } else {
#pragma unroll
                    for (int f = 0; f < NF; ++f) {
                        const T u = in_p[f * PL + po + r * WB];
                        y[r][f] = has_k ? rfma(a, in_p[(NF + f) * PL + po + r * WB], u) : u;
                    }
                }
            }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            w0[r][J] = y[r][0];
            if (NF > 1) w1[r][J] = y[r][NF - 1];
#pragma unroll
            for (int f = 0; f < NF; ++f) y_p[f * PL + po + r * WB] = y[r][f];
        }
        if (__syncthreads_or(!ok)) {
            failed = true;
            return false;
        }
        // the slot of plane p - RES is free (last read by step p-1): plane p + LA into it
        if (threadIdx.x == 0 && p + LA <= t_last) {
            m2::fence_proxy_async();
            issue(p + LA, si + LA < NS ? si + LA : si + LA - NS);
            issued = p + LA;
        }
        if (FINAL && sizeof(T) == 8 && threadIdx.x == 0 && A.pfm) {
            // k1, k2 and the low parts of the plane updated LA steps from now
            const int zp = p + LA - 2;
            if (zp >= z0 && zp < z1) {
                const int xq = x0 + gh - gh % G::VEC;
#pragma unroll
                for (int j = 0; j < 3; ++j)
#pragma unroll
                    for (int f = 0; f < NF; ++f)
                        if ((A.pfm >> (2 * j + f)) & 1) m2::tma_prefetch3(&A.tq[j][f], xq, y0 + gh, zp + gh);
            }
        }
        // ---- mu at plane p-1 on the tile + 1.  Every row of the thread is
        //      formed (rows off the tile + 1 read in-bounds values nobody uses and
        //      store them where nobody reads), so the rows interleave freely;
        //      with one row per thread, threads off the tile + 1 skip the phase
        //      (whole warps of the halo rows then issue nothing)
        if (DO_MU && (R > 1 || r1m)) {
            T muv[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const T cc = w0[r][J1];
                const T v2 = rmul((T)2, cc);
                T tx, ty;
                if (inner) {
                    const T* c = y_p1 + po + r * WB;
                    tx = second_diff(c[1], v2, c[-1]);
                    const T cn = r + 1 < R ? w0[r + 1 < R ? r + 1 : r][J1] : c[WB];
                    const T cs = r > 0 ? w0[r > 0 ? r - 1 : r][J1] : c[-WB];
                    ty = second_diff(cn, v2, cs);
                } else {
                    // the stencil centre: this cell, or the clamped cell on a zero-flux side
                    const int ly = ly0 + r, py = py0 + r;
                    int my = ly;
                    if (py < 0 && L.bc[2] == PHIX_BC_NOFLUX) my = -y0;
                    if (py >= n1 && L.bc[3] == PHIX_BC_NOFLUX) my = n1 - 1 - y0;
                    const T* c = y_p1 + po + r * WB + pmx + (my - ly) * WB;
                    tx = second_diff(c[1], v2, c[-1]);
                    ty = second_diff(c[WB], v2, c[-WB]);
                }
                const T tz = second_diff(w0[r][J], v2, w0[r][J2]);
                const T lap = lap_combine<T, 3>(tx, ty, tz, i2x, i2y, i2z);
                muv[r] = pol.mu(S, cc, lap, NF > 1 ? w1[r][J1] : (T)0);
            }
#pragma unroll
            for (int r = 0; r < R; ++r) {
                wm[r][J1] = muv[r];
                m_p1[po + r * WB] = muv[r];
            }
        }
        // (no barrier: the right-hand side reads mu of p-2 and y of p-2, both
        // stored before the barrier above)
        // ---- the right-hand side at plane p-2 on the tile: formed for every
        //      row of the thread, stored for the tile's rows
        if (DO_K && (R > 1 || tm)) {
            T kv[R][2];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int o = po + r * WB;
                const T* m = m_p2 + o;
                const T mv2 = rmul((T)2, wm[r][J2]);
                const T mtx = second_diff(m[1], mv2, m[-1]);
                const T mn = r + 1 < R ? wm[r + 1 < R ? r + 1 : r][J2] : m[WB];
                const T ms = r > 0 ? wm[r > 0 ? r - 1 : r][J2] : m[-WB];
                const T mty = second_diff(mn, mv2, ms);
                const T mtz = second_diff(wm[r][J1], mv2, wm[r][J3]);
                const T lapmu = lap_combine<T, 3>(mtx, mty, mtz, i2x, i2y, i2z);
                T lapy1 = (T)0;
                if (Pol::LAP_Y1) {
                    const T* e = y_p2 + (NF - 1) * PL + o;
                    const T ev2 = rmul((T)2, w1[r][J2]);
                    const T etx = second_diff(e[1], ev2, e[-1]);
                    const T en = r + 1 < R ? w1[r + 1 < R ? r + 1 : r][J2] : e[WB];
                    const T es = r > 0 ? w1[r > 0 ? r - 1 : r][J2] : e[-WB];
                    const T ety = second_diff(en, ev2, es);
                    const T etz = second_diff(w1[r][J1], ev2, w1[r][J3]);
                    lapy1 = lap_combine<T, 3>(etx, ety, etz, i2x, i2y, i2z);
                }
                pol.rhs(S, lapmu, w0[r][J2], (T)0, NF > 1 ? w1[r][J2] : (T)0, lapy1, kv[r]);
            }
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if (!((tm >> r) & 1u)) continue;
                [[maybe_unused]] const int o = po + r * WB;  // the update's slot offset
                const int idx = L.origin + gtile + s1 * r + s2 * z;
#pragma unroll
                for (int f = 0; f < NF; ++f) {
                    if constexpr (MODE == MODE_K) {
                        S.out[f][idx] = kv[r][f];
                    } else {
                        // emit's arithmetic, with u (and k3) from the plane's input slot
                        const T u = in_p2[f * PL + o];
                        T d;
                        if constexpr (MODE == MODE_RK4_FINAL) {
                            // phi += dt6 * (((k1 + 2 k2) + 2 k3) + k4)
                            T sum = radd(pk1[r][f], rmul((T)2, pk2[r][f]));
                            sum = radd(sum, rmul((T)2, in_p2[(NF + f) * PL + o]));
                            d = radd(sum, kv[r][f]);
                        } else {
                            d = kv[r][f];
                        }
                        if (S.ulo[f]) twosum_update(u, plo[r][f], rmul(S.dtf, d), &S.out[f][idx], &S.outlo[f][idx]);
                        else S.out[f][idx] = rfma(S.dtf, d, u);
                    }
                }
            }
        }
        si = si + 1 == NS ? 0 : si + 1;
        ph ^= si == 0 ? 1u : 0u;
        return true;
    };

    // ghost cells of the new state on planes za .. zb (the BC-mapped old state),
    // as stage_march3d writes them; once per group of planes, outside the plane
    // bodies, whose registers they would otherwise share
    auto ghosts = [&](const int za, const int zb) {
        for (int z = za; z <= zb; ++z) {
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
                        const int qxx = x0 + i % TX, l = 1 + i / TX;
                        if (qxx >= n0) continue;
                        if (y0 == 0) write_ghost<T, 3>(S, NF, qxx, -l, z);
                        if (y0 + TY >= n1) write_ghost<T, 3>(S, NF, qxx, n1 - 1 + l, z);
                    }
            }
            if (z == 0 || z == n2 - 1)
                for (int i = threadIdx.x; i < TX * TY * gh; i += G::NT) {
                    const int qxx = x0 + i % TX, qy = y0 + (i / TX) % TY, l = 1 + i / (TX * TY);
                    if (qxx >= n0 || qy >= n1) continue;
                    if (z == 0) write_ghost<T, 3>(S, NF, qxx, qy, -l);
                    if (z == n2 - 1) write_ghost<T, 3>(S, NF, qxx, qy, n2 - 1 + l);
                }
        }
    };

    // the march: planes z0-2 and z0-1 bring inputs only, z0 and z0+1 add mu,
    // then every plane forms mu and a right-hand side; four planes per pass so
    // that the ring positions are compile-time (t_last >= z0 + 2 always)
    using I0 = std::integral_constant<int, 0>;
    using I1 = std::integral_constant<int, 1>;
    using I2 = std::integral_constant<int, 2>;
    using I3 = std::integral_constant<int, 3>;
    using NO = std::false_type;
    using YES = std::true_type;
    if constexpr (!FINAL) {
        if (plane(I0{}, NO{}, NO{}, t_first) && plane(I1{}, NO{}, NO{}, t_first + 1) &&
            plane(I2{}, YES{}, NO{}, t_first + 2) && plane(I3{}, YES{}, NO{}, t_first + 3)) {
            for (int p = t_first + 4; p <= t_last; p += 4) {
                if (!plane(I0{}, YES{}, YES{}, p)) break;
                if (p + 1 > t_last || !plane(I1{}, YES{}, YES{}, p + 1)) break;
                if (p + 2 > t_last || !plane(I2{}, YES{}, YES{}, p + 2)) break;
                if (p + 3 > t_last || !plane(I3{}, YES{}, YES{}, p + 3)) break;
            }
        }
    } else {
        using IR = std::integral_constant<int, -1>;  // rolling
        if (plane(IR{}, NO{}, NO{}, t_first) && plane(IR{}, NO{}, NO{}, t_first + 1) &&
            plane(IR{}, YES{}, NO{}, t_first + 2) && plane(IR{}, YES{}, NO{}, t_first + 3)) {
            for (int p = t_first + 4; p <= t_last; ++p) {
                if (!plane(IR{}, YES{}, YES{}, p)) break;
                ghosts(p - 2, p - 2);
            }
        }
    }

    if (failed) {
        // a copy did not arrive in time: record it, and let the copies still in
        // flight land (bounded) before the CTA's shared memory is released
        if (threadIdx.x == 0) {
            atomicExch(A.err, 1);
            for (int t = max(issued - NS + 1, t_first); t <= issued; ++t)
                m2::bar_wait(bars + (t - t_first) % NS, (uint32_t)(((t - t_first) / NS) & 1), m2::WAIT_NS);
        }
        __syncthreads();
    }
}

}  // namespace phix
