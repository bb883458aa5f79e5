// march3d_fused.cuh -- 3-D RK4 of the chemical-potential physics (CH, coupled
// CH+AC) in two launches per time step, two stages fused in each.
//
//   launch A (stages 1, 2): k1 = F(u) on the tile + 2, y2 = u + dt/2 k1 there,
//                           k2 = F(y2) on the tile; writes k2 and
//                           acc = k1 + 2 k2 (the first two terms of the RK4 sum)
//   launch B (stages 3, 4): y3 = u + dt/2 k2 on the tile + 4, k3 = F(y3) on the
//                           tile + 2, y4 = u + dt k3, k4 = F(y4) on the tile;
//                           u' = u + dt/6 ((acc + 2 k3) + k4)
//
// (kernel_rk4_tmp / kernel_rk4_update, Solver.cu:49-71; VectorSolver.cu:149-228:
// every stage state gets the BCs, all components advance together.)
//
// Each CTA owns a TX x TY in-plane tile and marches a range of z planes.  The
// input planes (u, and k2 in launch B) arrive by TMA (cp.async.bulk.tensor,
// one box of (TX + 2E) x (TY + 2E) cells per plane and field, E = 4) into a
// ring of shared-memory slots, one mbarrier per slot, the next plane's copy in
// flight while the current plane is used.  All derived planes (mu of each
// stage, the stage states y2 / y4, and the tile's k of the first stage) live in
// shared-memory rings with the same row pitch, so no intermediate touches HBM.
// Software pipeline at step t (planes marching upwards):
//     input plane t lands          ->  mu_a(t-1) on the tile + 3
//     k_a(t-2), y_b(t-2) on the tile + 2  ->  mu_b(t-3) on the tile + 1
//     k_b(t-4) on the tile: outputs of plane t-4.
//
// Boundaries: z must be periodic (planes outside [0, n2) are read at their
// periodic image and the stages computed on the images, which gives the same
// bits); x and y sides may be periodic or zero-flux.  Input cells outside the
// grid are replaced after the copy by their BC-mapped values (map3).  Derived
// values outside the grid on a zero-flux side are computed at the clamped cell
// (mu_axis / map_axis semantics); on a periodic side they are computed on the
// images.  Every value sees the operations of stage_march3d in the same order
// (tile_lap, compute_mu, compute_rhs, the RK4 combination of emit), so the bits
// equal the four-launch path.
#pragma once

#include <cuda.h>
#include <stdint.h>

#include "phix/detail/stage.cuh"

namespace phix {

namespace m2 {

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_bar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// generic-proxy shared-memory accesses before a TMA write into the same bytes
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void arrive_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(b)), "r"(bytes) : "memory");
}
// One box of a 3-D tensor map into shared memory, completion on mbarrier b.
__device__ __forceinline__ void tma_box3(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* b) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(saddr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(saddr(b))
        : "memory");
}
// Prefetch one box of a 3-D tensor map into L2 (no shared memory, no completion).
__device__ __forceinline__ void tma_prefetch3(const CUtensorMap* map, int x, int y, int z) {
    asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y), "r"(z)
                 : "memory");
}
__device__ __forceinline__ bool bar_try_wait(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(saddr(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t now_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Wait for phase `parity` of b with a wall-clock limit; false = gave up.
__device__ __forceinline__ bool bar_wait(uint64_t* b, uint32_t parity, uint64_t limit_ns) {
    if (bar_try_wait(b, parity)) return true;
    const uint64_t t0 = now_ns();
    while (!bar_try_wait(b, parity))
        if (now_ns() - t0 > limit_ns) return false;
    return true;
}

// The same wait with the waiting thread suspended inside each try (up to
// 20 us, woken early when the phase completes) instead of spinning, so that
// it takes no issue slots from the CTA's other warps.
__device__ __forceinline__ bool bar_try_wait_sleep(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(saddr(b)), "r"(parity), "r"(20000u)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool bar_wait_sleep(uint64_t* b, uint32_t parity, uint64_t limit_ns) {
    if (bar_try_wait_sleep(b, parity)) return true;
    const uint64_t t0 = now_ns();
    while (!bar_try_wait_sleep(b, parity))
        if (now_ns() - t0 > limit_ns) return false;
    return true;
}

constexpr uint64_t WAIT_NS = 2000000000ull;  // a plane copy that takes 2 s has failed

}  // namespace m2

template <typename T>
struct March2Args {
    StageArgs<T> S;        // layout, u (and ulo / out / outlo in launch B), coefficients
    CUtensorMap tu[2];     // u of each field (box: WB x HB x 1)
    CUtensorMap tk[2];     // k2 of each field (launch B)
    T* k2[2];              // launch A writes, launch B reads (tile cells)
    T* acc[2];             // k1 + 2 k2: launch A writes, launch B reads
    T a_in;                // launch B: y3 = u + a_in k2 (dt/2)
    T a_mid;               // y_b = u + a_mid k_a (dt/2 in A, dt in B)
    int rz;                // output planes per CTA
    int* err;              // set when a plane copy did not arrive in time
};

template <typename T, class Pol, int TX, int TY, bool B>
struct March2 {
    static constexpr int NF = Pol::NF;
    static constexpr int E = 2 * Pol::H;                                  // input halo: two stages
    static constexpr int VEC = 16 / (int)sizeof(T);                       // TMA x granularity
    static constexpr int WB = (TX + 2 * E + VEC - 1 + VEC - 1) / VEC * VEC;  // plane row pitch = box width
    static constexpr int HB = TY + 2 * E;                                 // box rows
    static constexpr int PL = WB * HB;                                    // elements per plane slot
    static constexpr int TC = TX * TY;                                    // tile cells
    static constexpr int NU = B ? 6 : 5;   // u slots: planes t-4 (B) / t-3 .. t, and t+1 in flight
    static constexpr int NK2 = B ? 2 : 0;  // k2 slots (B): t and t+1
    static constexpr int NYA = B ? 4 : 0;  // y3 slots (B): t-3 .. t  (A reads u as y1)
    static constexpr int NM = 3;           // mu slots of each stage
    static constexpr int NKA = 3;          // k_a slots on the tile: t-4 .. t-2
    static constexpr int NYB = 4;          // y_b slots: t-5 .. t-2
    // slot sizes are multiples of 128 bytes (TMA destinations)
    static constexpr int PLA = (PL * (int)sizeof(T) + 127) / 128 * 128 / (int)sizeof(T);
    static constexpr size_t OFF_U = 0;
    static constexpr size_t OFF_K2 = OFF_U + (size_t)NU * NF * PLA;
    static constexpr size_t OFF_YA = OFF_K2 + (size_t)NK2 * NF * PLA;
    static constexpr size_t OFF_MA = OFF_YA + (size_t)NYA * NF * PLA;
    static constexpr size_t OFF_YB = OFF_MA + (size_t)NM * PLA;
    static constexpr size_t OFF_MB = OFF_YB + (size_t)NYB * NF * PLA;
    static constexpr size_t OFF_KA = OFF_MB + (size_t)NM * PLA;
    static constexpr size_t ELEMS = OFF_KA + (size_t)NKA * NF * TC;
    static constexpr size_t BAR_OFF = (ELEMS * sizeof(T) + 7) / 8 * 8;                   // mbarriers after the slots
    static constexpr size_t smem_bytes() { return 128 + BAR_OFF + (size_t)NU * 8; }  // + base alignment
    static constexpr uint32_t BOX_BYTES = (uint32_t)(PL * sizeof(T));
    static_assert(Pol::MU && Pol::H == 2, "the fused 3-D step is built for the chemical-potential physics");
    static_assert((WB * sizeof(T)) % 16 == 0, "box rows must be whole 16-byte units");
    static_assert(WB <= 256 && HB <= 256, "TMA box dimensions are at most 256");
};

template <typename T, class Pol, int TX, int TY, int NT, bool B>
__global__ void __launch_bounds__(NT) stage2_march3d(const __grid_constant__ March2Args<T> A) {
    using G = March2<T, Pol, TX, TY, B>;
    constexpr int NF = G::NF, E = G::E, WB = G::WB, HB = G::HB, PLA = G::PLA, TC = G::TC;
    constexpr int NU = G::NU, NM = G::NM, NKA = G::NKA, NYB = G::NYB;
    const Pol pol{};
    const StageArgs<T>& S = A.S;
    const Layout& L = S.L;
    // 128-byte aligned slots, offset from the shared array itself so that slot
    // accesses stay shared-memory accesses
    extern __shared__ __align__(128) unsigned char m2_raw[];
    T* sm = reinterpret_cast<T*>(m2_raw + ((128u - (m2::saddr(m2_raw) & 127u)) & 127u));
    uint64_t* bars = reinterpret_cast<uint64_t*>(reinterpret_cast<unsigned char*>(sm) + G::BAR_OFF);  // NU mbarriers

    const int n0 = L.n[0], n1 = L.n[1], n2 = L.n[2], gh = L.ghost;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int z0 = blockIdx.z * A.rz, z1 = min(z0 + A.rz, n2);
    constexpr int VEC = G::VEC;
    const int sh = ((gh - E) % VEC + VEC) % VEC;  // box starts on a 16-byte boundary
    const bool inner = x0 - E >= 0 && x0 + TX + E <= n0 && y0 - E >= 0 && y0 + TY + E <= n1;
    const bool nf_xl = L.bc[0] == PHIX_BC_NOFLUX, nf_xh = L.bc[1] == PHIX_BC_NOFLUX;
    const bool nf_yl = L.bc[2] == PHIX_BC_NOFLUX, nf_yh = L.bc[3] == PHIX_BC_NOFLUX;

    auto uslot = [&](int f, int z) -> T* { return sm + G::OFF_U + ((size_t)((unsigned)(z + 8 * NU) % NU) * NF + f) * PLA; };
    auto k2slot = [&](int f, int z) -> T* { return sm + G::OFF_K2 + ((size_t)((unsigned)(z + 8) % 2) * NF + f) * PLA; };
    auto yaslot = [&](int f, int z) -> T* {
        if constexpr (B) return sm + G::OFF_YA + ((size_t)((unsigned)(z + 8 * G::NYA) % G::NYA) * NF + f) * PLA;
        else return uslot(f, z);  // launch A: the first stage state is u itself
    };
    auto maslot = [&](int z) -> T* { return sm + G::OFF_MA + (size_t)((unsigned)(z + 8 * NM) % NM) * PLA; };
    auto ybslot = [&](int f, int z) -> T* { return sm + G::OFF_YB + ((size_t)((unsigned)(z + 8 * NYB) % NYB) * NF + f) * PLA; };
    auto mbslot = [&](int z) -> T* { return sm + G::OFF_MB + (size_t)((unsigned)(z + 8 * NM) % NM) * PLA; };
    auto kaslot = [&](int f, int z) -> T* { return sm + G::OFF_KA + ((size_t)((unsigned)(z + 8 * NKA) % NKA) * NF + f) * TC; };
    auto bar = [&](int z) -> uint64_t* { return bars + (unsigned)(z + 8 * NU) % NU; };

    // shared-memory offset of tile-relative cell (lx, ly), lx, ly in [-E, T + E)
    auto soff = [&](int lx, int ly) { return (lx + E + sh) + (ly + E) * WB; };
    // offset whose value cell (lx, ly) of a derived plane takes: itself, or on
    // a zero-flux side the clamped cell
    auto src_off = [&](int lx, int ly) {
        if (!inner) {
            const int px = x0 + lx, py = y0 + ly;
            if (px < 0 && nf_xl) lx = -x0;
            if (px >= n0 && nf_xh) lx = n0 - 1 - x0;
            if (py < 0 && nf_yl) ly = -y0;
            if (py >= n1 && nf_yh) ly = n1 - 1 - y0;
        }
        return soff(lx, ly);
    };
    auto zwrap = [&](int z) {
        if ((unsigned)z < (unsigned)n2) return z;
        const int r = z % n2;
        return r < 0 ? r + n2 : r;
    };

    // input planes z0 - E .. z1 + E - 1 (each stage reaches H = 2 planes)
    const int t_first = z0 - E, t_last = z1 + E - 1;
    auto issue = [&](int t) {  // thread 0: the input plane(s) of step t
        uint64_t* b = bar(t);
        m2::arrive_expect_tx(b, G::BOX_BYTES * NF * (B ? 2 : 1));
        const int xs = x0 - E + gh - sh, ys = y0 - E + gh, zs = zwrap(t) + gh;
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            m2::tma_box3(uslot(f, t), &A.tu[f], xs, ys, zs, b);
            if constexpr (B) m2::tma_box3(k2slot(f, t), &A.tk[f], xs, ys, zs, b);
        }
    };

    if (threadIdx.x == 0) {
        for (int i = 0; i < NU; ++i) m2::bar_init(bars + i, 1);
        m2::fence_bar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) issue(t_first);

    const T a_mid = A.a_mid;
    bool failed = false;
    int pending_last = t_first;  // last plane whose copy was issued

    for (int t = t_first; t <= t_last; ++t) {
        // ---- 1. input plane t: wait, BC-map the cells outside the grid,
        //         (launch B) form y3 = u + dt/2 k2
        const uint32_t parity = (uint32_t)(((t - t_first) / NU) & 1);
        const bool ok = m2::bar_wait(bar(t), parity, m2::WAIT_NS);
        if (__syncthreads_or(!ok)) { failed = true; break; }
        if (!inner) {
            const int zw = zwrap(t);
            for (int i = threadIdx.x; i < (TX + 2 * E) * HB; i += NT) {
                const int lx = i % (TX + 2 * E) - E, ly = i / (TX + 2 * E) - E;
                const int px = x0 + lx, py = y0 + ly;
                if (px >= 0 && px < n0 && py >= 0 && py < n1) continue;
                int idx;
                double cval;
                map3<3>(L, px, py, zw, &idx, &cval);  // periodic / zero-flux sides: never constant
                const int o = soff(lx, ly);
#pragma unroll
                for (int f = 0; f < NF; ++f) {
                    uslot(f, t)[o] = __ldg(S.u[f] + idx);
                    if constexpr (B) k2slot(f, t)[o] = __ldg(A.k2[f] + idx);
                }
            }
            if constexpr (B) __syncthreads();
        }
        if constexpr (B) {
            const T a_in = A.a_in;
            for (int i = threadIdx.x; i < PLA; i += NT)
#pragma unroll
                for (int f = 0; f < NF; ++f) yaslot(f, t)[i] = rfma(a_in, k2slot(f, t)[i], uslot(f, t)[i]);
        }
        __syncthreads();
        // ---- 2. the next plane's copy (its slot was last read before the barrier above)
        if (threadIdx.x == 0 && t + 1 <= t_last) {
            m2::fence_proxy_async();
            issue(t + 1);
            pending_last = t + 1;
        }
        // ---- 3. mu of the first stage at plane t-1, on the tile + E - 1
        {
            const int z = t - 1;
            if (z >= t_first + 1 && z <= t_last - 1) {
                constexpr int RW = TX + 2 * (E - 1), RH = TY + 2 * (E - 1);
                T* dst = maslot(z);
                const T* yc0 = yaslot(0, z);
                const T* ym0 = yaslot(0, z - 1);
                const T* yp0 = yaslot(0, z + 1);
                const T* yc1 = yaslot(NF - 1, z);
                for (int i = threadIdx.x; i < RW * RH; i += NT) {
                    const int lx = i % RW - (E - 1), ly = i / RW - (E - 1);
                    dst[soff(lx, ly)] = compute_mu<T, Pol, 3, WB>(S, pol, yc0, ym0, yp0, yc1, src_off(lx, ly));
                }
            }
        }
        __syncthreads();
        // ---- 4. k of the first stage at plane t-2 on the tile + E - 2;
        //         y_b = u + a_mid k_a there; k_a of the tile cells kept
        {
            const int z = t - 2;
            if (z >= t_first + 2 && z <= t_last - 2) {
                constexpr int RW = TX + 2 * (E - 2), RH = TY + 2 * (E - 2);
                const T *mc = maslot(z), *mm = maslot(z - 1), *mp = maslot(z + 1);
                const T *y0c = yaslot(0, z), *y0m = yaslot(0, z - 1), *y0p = yaslot(0, z + 1);
                const T *y1c = yaslot(NF - 1, z), *y1m = yaslot(NF - 1, z - 1), *y1p = yaslot(NF - 1, z + 1);
                for (int i = threadIdx.x; i < RW * RH; i += NT) {
                    const int lx = i % RW - (E - 2), ly = i / RW - (E - 2);
                    const int so = src_off(lx, ly), o = soff(lx, ly);
                    T k[2];
                    compute_rhs<T, Pol, 3, WB, WB>(S, pol, mc, mm, mp, so, y0c, y0m, y0p, y1c, y1m, y1p, so, k);
#pragma unroll
                    for (int f = 0; f < NF; ++f) ybslot(f, z)[o] = rfma(a_mid, k[f], uslot(f, z)[so]);
                    if (lx >= 0 && lx < TX && ly >= 0 && ly < TY)
#pragma unroll
                        for (int f = 0; f < NF; ++f) kaslot(f, z)[lx + ly * TX] = k[f];
                }
            }
        }
        __syncthreads();
        // ---- 5. mu of the second stage at plane t-3, on the tile + 1
        {
            const int z = t - 3;
            if (z >= t_first + 3 && z <= t_last - 3) {
                constexpr int RW = TX + 2, RH = TY + 2;
                T* dst = mbslot(z);
                const T* yc0 = ybslot(0, z);
                const T* ym0 = ybslot(0, z - 1);
                const T* yp0 = ybslot(0, z + 1);
                const T* yc1 = ybslot(NF - 1, z);
                for (int i = threadIdx.x; i < RW * RH; i += NT) {
                    const int lx = i % RW - 1, ly = i / RW - 1;
                    dst[soff(lx, ly)] = compute_mu<T, Pol, 3, WB>(S, pol, yc0, ym0, yp0, yc1, src_off(lx, ly));
                }
            }
        }
        __syncthreads();
        // ---- 6. k of the second stage at plane t-4 on the tile: the outputs
        {
            const int z = t - 4;
            if (z >= z0 && z < z1) {
                const T *mc = mbslot(z), *mm = mbslot(z - 1), *mp = mbslot(z + 1);
                const T *y0c = ybslot(0, z), *y0m = ybslot(0, z - 1), *y0p = ybslot(0, z + 1);
                const T *y1c = ybslot(NF - 1, z), *y1m = ybslot(NF - 1, z - 1), *y1p = ybslot(NF - 1, z + 1);
                const int zidx = L.origin + L.s[2] * z;
                for (int i = threadIdx.x; i < TC; i += NT) {
                    const int lx = i % TX, ly = i / TX;
                    const int px = x0 + lx, py = y0 + ly;
                    if (px >= n0 || py >= n1) continue;
                    const int o = soff(lx, ly);
                    T k[2];
                    compute_rhs<T, Pol, 3, WB, WB>(S, pol, mc, mm, mp, o, y0c, y0m, y0p, y1c, y1m, y1p, o, k);
                    const int idx = zidx + px + L.s[1] * py;
#pragma unroll
                    for (int f = 0; f < NF; ++f) {
                        const T ka = kaslot(f, z)[i];
                        if constexpr (!B) {
                            A.k2[f][idx] = k[f];
                            A.acc[f][idx] = radd(ka, rmul((T)2, k[f]));  // k1 + 2 k2
                        } else {
                            // phi += dt6 * (((k1 + 2 k2) + 2 k3) + k4)
                            T s = radd(__ldg(A.acc[f] + idx), rmul((T)2, ka));
                            s = radd(s, k[f]);
                            const T u = uslot(f, z)[o];
                            if (S.ulo[f]) {
                                twosum_update(u, __ldg(S.ulo[f] + idx), rmul(S.dtf, s), &S.out[f][idx],
                                              &S.outlo[f][idx]);
                            } else {
                                S.out[f][idx] = rfma(S.dtf, s, u);
                            }
                        }
                    }
                }
                if constexpr (B) {
                    // ghost cells of the new state (the BC-mapped old state), as stage_march3d writes them
                    if (!inner) {
                        if (x0 == 0 || x0 + TX >= n0)
                            for (int i = threadIdx.x; i < TY * gh; i += NT) {
                                const int py = y0 + i / gh, l = 1 + i % gh;
                                if (py >= n1) continue;
                                if (x0 == 0) write_ghost<T, 3>(S, NF, -l, py, z);
                                if (x0 + TX >= n0) write_ghost<T, 3>(S, NF, n0 - 1 + l, py, z);
                            }
                        if (y0 == 0 || y0 + TY >= n1)
                            for (int i = threadIdx.x; i < TX * gh; i += NT) {
                                const int px = x0 + i % TX, l = 1 + i / TX;
                                if (px >= n0) continue;
                                if (y0 == 0) write_ghost<T, 3>(S, NF, px, -l, z);
                                if (y0 + TY >= n1) write_ghost<T, 3>(S, NF, px, n1 - 1 + l, z);
                            }
                    }
                    if (z == 0 || z == n2 - 1)
                        for (int i = threadIdx.x; i < TC * gh; i += NT) {
                            const int lx = i % TX, ly = (i / TX) % TY, l = 1 + i / TC;
                            const int px = x0 + lx, py = y0 + ly;
                            if (px >= n0 || py >= n1) continue;
                            if (z == 0) write_ghost<T, 3>(S, NF, px, py, -l);
                            if (z == n2 - 1) write_ghost<T, 3>(S, NF, px, py, n2 - 1 + l);
                        }
                }
            }
        }
        // step t+1 writes only slots whose last readers finished before one of
        // the barriers above or the one after its own wait
    }

    if (failed) {
        // a copy did not arrive in time: record it, and let the copies still in
        // flight land (bounded) before the CTA's shared memory is released
        if (threadIdx.x == 0) {
            atomicExch(A.err, 1);
            for (int t = pending_last - NU + 1; t <= pending_last; ++t) {
                if (t < t_first) continue;
                m2::bar_wait(bar(t), (uint32_t)(((t - t_first) / NU) & 1), m2::WAIT_NS);
            }
        }
        __syncthreads();
    }
}

}  // namespace phix
