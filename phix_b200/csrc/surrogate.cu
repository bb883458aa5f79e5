// surrogate.cu -- learned Cahn-Hilliard surrogate: a 4-layer 3x3 CNN
// (1 -> 32 -> 32 -> 32 -> 1, GELU, circular padding) that advances c by 50
// FD time steps, followed by an exact FP64 mean-mass projection.
//
// The two 32 -> 32 layers carry 97% of the FLOPs and run on the 5th-gen
// tensor cores as implicit GEMMs (tcgen05.mma kind::f16, BF16 operands from
// shared memory, FP32 accumulator in TMEM):
//   forward / data-gradient : M = 128 output pixels of one row, N = 32
//       channels, K = 9 taps x 32 channels = 18 MMAs of K = 16.  The three
//       input rows are staged once per tile as [chunk][pixel][8] (K-major,
//       no swizzle); each tap is the same buffer at a shifted start address.
//       Epilogue: + bias, GELU, BF16 store (forward) or x GELU'(z) (data
//       gradient, with the weights flipped and transposed).
//   weight gradient         : per 16-pixel K step, three MMAs (one per dx)
//       with M = 128 = (4 staged rows x 32 input channels) and N = 32
//       output channels, both operands MN-major; accumulators stay in TMEM
//       for all tiles of the CTA, partial sums per CTA are reduced in a fixed
//       order.
// The 1 -> 32 and 32 -> 1 layers (3% of the FLOPs), the loss, Adam and the
// projection run on CUDA cores.  Activations are NHWC BF16 [B][H][W][32].
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "phix/detail/common.cuh"
#include "stepper.h"
#include "tc_sm100.cuh"

namespace phix {
namespace sg {

constexpr int CH = 32;
constexpr int TILE = 128;   // output pixels per tile (one row segment)
constexpr int NT = 128;     // 4 warps: one per TMEM lane quadrant
constexpr int HALO_PX = TILE + 2;
constexpr int CHUNK_B = HALO_PX * 16;  // 2080: one 8-channel chunk of a staged row
constexpr int ROW_B = 4 * CHUNK_B;     // 8320: one staged row, 32 channels
constexpr int WPK_B = 9 * 2 * 1024;    // packed weights: (tap, k16) blocks of [2][32][8] bf16
constexpr int DROW_B = 4 * TILE * 16;  // 8192: one un-haloed row (weight-gradient B operand)
constexpr uint64_t WAIT_NS = 2000000000ull;  // give up on an mbarrier after 2 s
constexpr int WGRAD_SMEM = 56 * 1024;         // >= 4 * ROW_B + DROW_B + 16; caps residency at 4 CTAs/SM

__device__ __forceinline__ float gelu_f(float x) {
    const float k = 0.7978845608028654f, c = 0.044715f;
    return 0.5f * x * (1.0f + tanhf(k * (x + c * x * x * x)));
}
__device__ __forceinline__ float gelu_grad_f(float x) {
    const float k = 0.7978845608028654f, c = 0.044715f;
    const float t = tanhf(k * (x + c * x * x * x));
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * k * (1.0f + 3.0f * c * x * x);
}

__device__ __forceinline__ uint32_t pack2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}
__device__ __forceinline__ void unpack8(uint4 u, float* f) {
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        float2 v = __bfloat1622float2(h[i]);
        f[2 * i] = v.x;
        f[2 * i + 1] = v.y;
    }
}

__device__ __forceinline__ int wrap(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// Stage `nrows` input rows y-1 .. y-2+nrows, pixels x0-1 .. x0+TILE, as
// [row][chunk][pixel][8 channels] (16-byte units, circular wrap).
__device__ __forceinline__ void stage_rows(uint8_t* rows, const __nv_bfloat16* __restrict__ x, int b, int y, int x0,
                                           int H, int W, int nrows) {
    const int units = nrows * HALO_PX * 4;
    for (int u = threadIdx.x; u < units; u += NT) {
        const int r = u / (HALO_PX * 4), rem = u - r * HALO_PX * 4, i = rem >> 2, j = rem & 3;
        const int gy = wrap(y + r - 1, H), gx = wrap(x0 - 1 + i, W);
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(x + (((size_t)b * H + gy) * W + gx) * CH) + j);
        *reinterpret_cast<uint4*>(rows + r * ROW_B + j * CHUNK_B + i * 16) = v;
    }
}

struct ConvArgs {
    const __nv_bfloat16* x;     // [B][H][W][32]
    const __nv_bfloat16* wpk;   // packed weights (WPK_B bytes)
    const float* bias;          // [32] (forward)
    const __nv_bfloat16* zaux;  // data gradient: pre-activation whose GELU' scales the output
    __nv_bfloat16* out;         // forward: gelu(z); data gradient: dz
    __nv_bfloat16* zout;        // forward: z (may be null)
    int B, H, W;
    int* err;
};

enum : int { EPI_FWD = 0, EPI_DGRAD = 1 };

template <int EPI>
__global__ void __launch_bounds__(NT) conv32_tc(const ConvArgs a) {
    extern __shared__ __align__(1024) uint8_t sm[];
    uint8_t* wbuf = sm;
    uint8_t* rows = sm + WPK_B;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + WPK_B + 3 * ROW_B);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    for (int u = threadIdx.x; u < WPK_B / 16; u += NT)
        reinterpret_cast<uint4*>(wbuf)[u] = __ldg(reinterpret_cast<const uint4*>(a.wpk) + u);
    if (warp == 0) {
        tc::tmem_alloc(slot, 32);
        tc::tmem_relinquish();
    }
    if (threadIdx.x == 0) tc::mbar_init(bar, 1);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *slot;
    const uint32_t idesc = tc::idesc_bf16_f32(128, 32, 0, 0);
    const uint32_t rows_a = tc::smem_u32(rows), w_a = tc::smem_u32(wbuf);

    const int tpr = a.W / TILE;
    const int ntiles = a.B * a.H * tpr;
    uint32_t phase = 0;
    bool failed = false;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int b = t / (a.H * tpr), rem = t - b * a.H * tpr, y = rem / tpr, x0 = (rem - y * tpr) * TILE;
        stage_rows(rows, a.x, b, y, x0, a.H, a.W, 3);
        tc::fence_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
            tc::fence_after_sync();
#pragma unroll
            for (int tap = 0; tap < 9; ++tap)
#pragma unroll
                for (int kk = 0; kk < 2; ++kk) {
                    const int ky = tap / 3, kx = tap % 3;
                    const uint64_t ad = tc::sdesc(rows_a + ky * ROW_B + 2 * kk * CHUNK_B + kx * 16, CHUNK_B, 128);
                    const uint64_t bd = tc::sdesc(w_a + (tap * 2 + kk) * 1024, 512, 128);
                    tc::umma_bf16(tmem, ad, bd, idesc, (tap | kk) != 0);
                }
            tc::umma_commit(bar);
        }
        if (!tc::mbar_wait_bounded(bar, phase, WAIT_NS)) {
            failed = true;
            break;
        }
        phase ^= 1u;
        tc::fence_after_sync();
        float v[32];
        tc::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16), v);
        const int gx = x0 + warp * 32 + lane;
        const size_t o = (((size_t)b * a.H + y) * a.W + gx) * CH;
        uint4* dst = reinterpret_cast<uint4*>(a.out + o);
        if (EPI == EPI_FWD) {
#pragma unroll
            for (int n = 0; n < 32; ++n) v[n] += __ldg(a.bias + n);
            if (a.zout) {
                uint4* zd = reinterpret_cast<uint4*>(a.zout + o);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    zd[q] = make_uint4(pack2(v[8 * q], v[8 * q + 1]), pack2(v[8 * q + 2], v[8 * q + 3]),
                                       pack2(v[8 * q + 4], v[8 * q + 5]), pack2(v[8 * q + 6], v[8 * q + 7]));
            }
#pragma unroll
            for (int n = 0; n < 32; ++n) v[n] = gelu_f(v[n]);
        } else {
            const uint4* zp = reinterpret_cast<const uint4*>(a.zaux + o);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float zf[8];
                unpack8(__ldg(zp + q), zf);
#pragma unroll
                for (int e = 0; e < 8; ++e) v[8 * q + e] *= gelu_grad_f(zf[e]);
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
            dst[q] = make_uint4(pack2(v[8 * q], v[8 * q + 1]), pack2(v[8 * q + 2], v[8 * q + 3]),
                                pack2(v[8 * q + 4], v[8 * q + 5]), pack2(v[8 * q + 6], v[8 * q + 7]));
        tc::fence_before_sync();
        __syncthreads();
    }
    if (failed && threadIdx.x == 0) atomicExch(a.err, 1);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 32);
}

// ---------------------------------------------------------------------------
// Forward 32 -> 32 convolution, row-pipelined.  A CTA owns strips of
// `rows` consecutive output rows of one 128-pixel column segment and walks
// them top to bottom with a ring of 6 staged input rows: each output row
// stages one new input row (cp.async, issued two rows ahead), the 18 UMMAs of
// row y run into TMEM accumulator y&1 while the epilogue (bias, GELU, BF16
// store) of row y-1 drains the other accumulator.  Same arithmetic as
// conv32_tc<EPI_FWD> except GELU's tanh, which uses the hardware tanh.approx
// instruction.
// ---------------------------------------------------------------------------
constexpr int RING = 6;
constexpr int NT_ROWS = 256;  // 8 warps: warp w drains TMEM lanes 32*(w%4).. and channels 16*(w/4)..

__device__ __forceinline__ void cp_async16(uint32_t saddr, const void* g) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

__device__ __forceinline__ float tanh_hw(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float gelu_hw(float x) {
    const float k = 0.7978845608028654f, c = 0.044715f;
    return 0.5f * x * (1.0f + tanh_hw(k * (x + c * x * x * x)));
}

// Stage input row gy (wrapped) of image b, pixels x0-1 .. x0+TILE, into ring slot `slot`
// (cp.async by the NTH threads of the CTA).
template <int NTH = NT_ROWS>
__device__ __forceinline__ void stage_row_async(uint32_t rows_a, int slot, const __nv_bfloat16* __restrict__ x, int b,
                                                int gy, int x0, int H, int W) {
    gy = wrap(gy, H);
    const __nv_bfloat16* src = x + ((size_t)b * H + gy) * W * CH;
#pragma unroll
    for (int u = threadIdx.x; u < HALO_PX * 4; u += NTH) {
        const int i = u >> 2, j = u & 3;
        const int gx = wrap(x0 - 1 + i, W);
        cp_async16(rows_a + slot * ROW_B + j * CHUNK_B + i * 16, src + (size_t)gx * CH + j * 8);
    }
}

__global__ void __launch_bounds__(NT_ROWS) conv32_rows_tc(const ConvArgs a, int rows) {
    extern __shared__ __align__(1024) uint8_t sm[];
    uint8_t* wbuf = sm;
    uint8_t* ring = sm + WPK_B;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + WPK_B + RING * ROW_B);  // 2 barriers
    uint32_t* slot_t = reinterpret_cast<uint32_t*>(bar + 2);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    for (int u = threadIdx.x; u < WPK_B / 16; u += NT_ROWS)
        reinterpret_cast<uint4*>(wbuf)[u] = __ldg(reinterpret_cast<const uint4*>(a.wpk) + u);
    if (warp == 0) {
        tc::tmem_alloc(slot_t, 64);
        tc::tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        tc::mbar_init(bar, 1);
        tc::mbar_init(bar + 1, 1);
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *slot_t;
    const uint32_t idesc = tc::idesc_bf16_f32(128, 32, 0, 0);
    const uint32_t ring_a = tc::smem_u32(ring), w_a = tc::smem_u32(wbuf);
    const int quad = warp & 3, half = warp >> 2;  // TMEM lane quadrant, channel half
    float bias[16];
#pragma unroll
    for (int n = 0; n < 16; ++n) bias[n] = __ldg(a.bias + 16 * half + n);

    const int tpr = a.W / TILE;
    const int nstrips = (a.H + rows - 1) / rows;
    const int njobs = a.B * tpr * nstrips;
    uint32_t phase[2] = {0u, 0u};
    bool failed = false;
    for (int job = blockIdx.x; job < njobs && !failed; job += gridDim.x) {
        const int b = job / (tpr * nstrips), rem = job - b * tpr * nstrips;
        const int strip = rem / tpr, x0 = (rem - strip * tpr) * TILE;
        const int y0 = strip * rows, y1 = min(y0 + rows, a.H);
        // rows y0-1, y0, y0+1 -> slots 0, 1, 2 (slot of row r: (r - y0 + 1) % RING),
        // then y0+2 as its own group (two rows in flight ahead of the UMMAs)
        for (int r = 0; r < 3; ++r) stage_row_async(ring_a, r, a.x, b, y0 - 1 + r, x0, a.H, a.W);
        cp_async_commit();
        if (y0 + 2 <= y1) stage_row_async(ring_a, 3, a.x, b, y0 + 2, x0, a.H, a.W);
        cp_async_commit();
        auto epilogue = [&](int y) {
            const int acc = y & 1;
            if (!tc::mbar_wait_bounded(bar + acc, phase[acc], WAIT_NS)) {
                failed = true;
                return;
            }
            phase[acc] ^= 1u;
            tc::fence_after_sync();
            float v[16];
            tc::tmem_ld16(tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(acc * 32 + 16 * half), v);
            const int gx = x0 + quad * 32 + lane;
            const size_t o = (((size_t)b * a.H + y) * a.W + gx) * CH + 16 * half;
#pragma unroll
            for (int n = 0; n < 16; ++n) v[n] += bias[n];
            if (a.zout) {
                uint4* zd = reinterpret_cast<uint4*>(a.zout + o);
#pragma unroll
                for (int q = 0; q < 2; ++q)
                    zd[q] = make_uint4(pack2(v[8 * q], v[8 * q + 1]), pack2(v[8 * q + 2], v[8 * q + 3]),
                                       pack2(v[8 * q + 4], v[8 * q + 5]), pack2(v[8 * q + 6], v[8 * q + 7]));
            }
#pragma unroll
            for (int n = 0; n < 16; ++n) v[n] = gelu_hw(v[n]);
            uint4* dst = reinterpret_cast<uint4*>(a.out + o);
#pragma unroll
            for (int q = 0; q < 2; ++q)
                dst[q] = make_uint4(pack2(v[8 * q], v[8 * q + 1]), pack2(v[8 * q + 2], v[8 * q + 3]),
                                    pack2(v[8 * q + 4], v[8 * q + 5]), pack2(v[8 * q + 6], v[8 * q + 7]));
        };
        for (int y = y0; y < y1; ++y) {
            // rows y-1 .. y+1 resident (this thread's copies, then everyone's;
            // the newest group, row y+2, may still be in flight); a timed-out
            // wait anywhere in the CTA stops every thread here
            cp_async_wait_one();
            tc::fence_async_smem();
            tc::fence_before_sync();
            if (__syncthreads_or(failed)) {
                failed = true;
                break;
            }
            tc::fence_after_sync();
            if (threadIdx.x == 0) {
                const int acc = y & 1;
#pragma unroll
                for (int tap = 0; tap < 9; ++tap)
#pragma unroll
                    for (int kk = 0; kk < 2; ++kk) {
                        const int ky = tap / 3, kx = tap % 3;
                        const int slot = (y - 1 + ky - y0 + 1) % RING;
                        const uint64_t ad =
                            tc::sdesc(ring_a + slot * ROW_B + 2 * kk * CHUNK_B + kx * 16, CHUNK_B, 128);
                        const uint64_t bd = tc::sdesc(w_a + (tap * 2 + kk) * 1024, 512, 128);
                        tc::umma_bf16(tmem + (uint32_t)(acc * 32), ad, bd, idesc, (tap | kk) != 0);
                    }
                tc::umma_commit(bar + acc);
            }
            // input row y+3 into the slot of row y-3 (its last reader, row y-2's
            // UMMAs, completed before row y-2's epilogue ran in the previous
            // iteration); an empty group keeps the group count uniform
            if (y + 3 <= y1) stage_row_async(ring_a, (y + 3 - y0 + 1) % RING, a.x, b, y + 3, x0, a.H, a.W);
            cp_async_commit();
            if (y > y0) epilogue(y - 1);
        }
        if (!failed) epilogue(y1 - 1);
        // the ring is reused by the next strip
        cp_async_wait_all();
        tc::fence_before_sync();
        failed = __syncthreads_or(failed);
        tc::fence_after_sync();
    }
    if (failed && threadIdx.x == 0) atomicExch(a.err, 1);
    cp_async_wait_all();
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 64);
}

struct WgradArgs {
    const __nv_bfloat16* x;   // layer input [B][H][W][32]
    const __nv_bfloat16* dz;  // gradient w.r.t. the layer's pre-activation
    float* partial;           // [gridDim.x][32 n][9 taps][32 ci]
    int B, H, W;
    int* err;
};

__global__ void __launch_bounds__(NT) conv32_wgrad_tc(const WgradArgs a) {
    extern __shared__ __align__(1024) uint8_t sm[];
    uint8_t* rows = sm;                        // 4 staged rows (the 4th only pads M to 128)
    uint8_t* drow = sm + 4 * ROW_B;            // [chunk][pixel][8] of dz, row y
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + 4 * ROW_B + DROW_B);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        tc::tmem_alloc(slot, 128);
        tc::tmem_relinquish();
    }
    if (threadIdx.x == 0) tc::mbar_init(bar, 1);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *slot;
    const uint32_t idesc = tc::idesc_bf16_f32(128, 32, 1, 1);
    const uint32_t rows_a = tc::smem_u32(rows), d_a = tc::smem_u32(drow);
    const int tpr = a.W / TILE;
    const int ntiles = a.B * a.H * tpr;
    uint32_t phase = 0;
    bool failed = false, any = false;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int b = t / (a.H * tpr), rem = t - b * a.H * tpr, y = rem / tpr, x0 = (rem - y * tpr) * TILE;
        stage_rows(rows, a.x, b, y, x0, a.H, a.W, 4);
        for (int u = threadIdx.x; u < TILE * 4; u += NT) {
            const int i = u >> 2, j = u & 3;
            const uint4 v =
                __ldg(reinterpret_cast<const uint4*>(a.dz + (((size_t)b * a.H + y) * a.W + x0 + i) * CH) + j);
            *reinterpret_cast<uint4*>(drow + j * (TILE * 16) + i * 16) = v;
        }
        tc::fence_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
            tc::fence_after_sync();
#pragma unroll
            for (int k = 0; k < TILE / 16; ++k)
#pragma unroll
                for (int dx = 0; dx < 3; ++dx) {
                    const uint64_t ad = tc::sdesc(rows_a + (16 * k + dx) * 16, 128, CHUNK_B);
                    const uint64_t bd = tc::sdesc(d_a + 16 * k * 16, 128, TILE * 16);
                    tc::umma_bf16(tmem + dx * 32, ad, bd, idesc, (any || k > 0) ? 1u : 0u);
                }
            tc::umma_commit(bar);
        }
        any = true;
        if (!tc::mbar_wait_bounded(bar, phase, WAIT_NS)) {
            failed = true;
            break;
        }
        phase ^= 1u;
        tc::fence_before_sync();
        __syncthreads();  // staged rows are overwritten by the next tile
    }
    tc::fence_after_sync();
    float* part = a.partial + (size_t)blockIdx.x * (32 * 9 * 32);
    if (!failed && warp < 3) {
        // D_dx row r*32 + ci (r = ky), column n
        for (int dx = 0; dx < 3; ++dx) {
            float v[32];
            if (any) {
                tc::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + dx * 32, v);
            } else {
#pragma unroll
                for (int n = 0; n < 32; ++n) v[n] = 0.f;
            }
            const int tap = warp * 3 + dx;
#pragma unroll
            for (int n = 0; n < 32; ++n) part[(n * 9 + tap) * 32 + lane] = v[n];
        }
    }
    if (failed && threadIdx.x == 0) atomicExch(a.err, 1);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 128);
}

// out[i] = sum_b partial[b][i] in block order (deterministic); i < n.
__global__ void reduce_partials(const float* __restrict__ partial, int nblocks, int n, float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float s = 0.f;
    for (int b = 0; b < nblocks; ++b) s += partial[(size_t)b * n + i];
    out[i] = s;
}

// ---------------------------------------------------------------------------
// CUDA-core layers
// ---------------------------------------------------------------------------
struct NetParams {
    double in_shift, in_scale, out_scale;
};

__device__ __forceinline__ float x0_at(const double* c, int b, int y, int x, int H, int W, NetParams P) {
    const double v = (c[((size_t)b * H + y) * W + x] - P.in_shift) * P.in_scale;
    return __bfloat162float(__float2bfloat16_rn((float)v));
}

// Layer 1: 1 -> 32.  w1 [32 n][9 taps] (bf16-rounded floats), b1 [32].
__global__ void __launch_bounds__(256) layer1_fwd(const double* __restrict__ c, const float* __restrict__ w1,
                                                  const float* __restrict__ b1, __nv_bfloat16* __restrict__ z1,
                                                  __nv_bfloat16* __restrict__ h1, int B, int H, int W, NetParams P) {
    __shared__ float ws[32 * 9], bs[32];
    for (int i = threadIdx.x; i < 32 * 9; i += 256) ws[i] = w1[i];
    if (threadIdx.x < 32) bs[threadIdx.x] = b1[threadIdx.x];
    __syncthreads();
    const size_t N = (size_t)B * H * W;
    for (size_t p = blockIdx.x * 256ull + threadIdx.x; p < N; p += (size_t)gridDim.x * 256) {
        const int b = (int)(p / ((size_t)H * W)), y = (int)((p / W) % H), x = (int)(p % W);
        float xv[9];
#pragma unroll
        for (int t = 0; t < 9; ++t) xv[t] = x0_at(c, b, wrap(y + t / 3 - 1, H), wrap(x + t % 3 - 1, W), H, W, P);
        uint4* zd = reinterpret_cast<uint4*>(z1 + p * CH);
        uint4* hd = reinterpret_cast<uint4*>(h1 + p * CH);
        for (int q = 0; q < 4; ++q) {  // one 8-channel group at a time
            float z[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const int n = 8 * q + e;
                float s = 0.f;
#pragma unroll
                for (int t = 0; t < 9; ++t) s = fmaf(xv[t], ws[n * 9 + t], s);
                z[e] = s + bs[n];
            }
            if (z1) zd[q] = make_uint4(pack2(z[0], z[1]), pack2(z[2], z[3]), pack2(z[4], z[5]), pack2(z[6], z[7]));
            hd[q] = make_uint4(pack2(gelu_hw(z[0]), gelu_hw(z[1])), pack2(gelu_hw(z[2]), gelu_hw(z[3])),
                               pack2(gelu_hw(z[4]), gelu_hw(z[5])), pack2(gelu_hw(z[6]), gelu_hw(z[7])));
        }
    }
}

// Layer 4: 32 -> 1 and the state update  c_out = c + out_scale * o.
// w4 [9 taps][32 ci], b4 [1].  Per-block FP64 partial sums of c and c_out per
// image go to part[(blockIdx, image)] for the mean-mass projection; o is also
// written when `o_out` is non-null (training).
__global__ void __launch_bounds__(256) layer4_fwd(const __nv_bfloat16* __restrict__ h3, const float* __restrict__ w4,
                                                  const float* __restrict__ b4, const double* __restrict__ c,
                                                  double* __restrict__ c_out, float* __restrict__ o_out, int B, int H,
                                                  int W, NetParams P) {
    __shared__ float ws[9 * 32];
    for (int i = threadIdx.x; i < 9 * 32; i += 256) ws[i] = w4[i];
    __syncthreads();
    const size_t N = (size_t)B * H * W;
    for (size_t p = blockIdx.x * 256ull + threadIdx.x; p < N; p += (size_t)gridDim.x * 256) {
        const int b = (int)(p / ((size_t)H * W)), y = (int)((p / W) % H), x = (int)(p % W);
        float s = 0.f;
#pragma unroll
        for (int t = 0; t < 9; ++t) {
            const size_t q = (((size_t)b * H + wrap(y + t / 3 - 1, H)) * W + wrap(x + t % 3 - 1, W)) * CH;
            const uint4* src = reinterpret_cast<const uint4*>(h3 + q);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                float f[8];
                unpack8(__ldg(src + k), f);
#pragma unroll
                for (int e = 0; e < 8; ++e) s = fmaf(f[e], ws[t * 32 + 8 * k + e], s);
            }
        }
        const float o = s + b4[0];
        if (o_out) o_out[p] = o;
        if (c_out) c_out[p] = c[p] + P.out_scale * (double)o;
    }
}

// Layer 4 on 128-pixel row segments staged in shared memory (3 input rows,
// [row][chunk][pixel][8 channels], circular wrap).  Block (bx, image) takes a
// contiguous range of the image's segments ordered segment-major, so
// consecutive segments are consecutive rows and each one stages a single new
// row.  Also writes c_out = c + out_scale * o and this block's FP64 sums of c
// and c_out to part[(image * gridDim.x + bx) * 2 + {0, 1}] for the mass
// projection (fixed order, so the result is deterministic).
constexpr int L4_MAXBLK = 2048;

__global__ void __launch_bounds__(NT) layer4_rows(const __nv_bfloat16* __restrict__ h3, const float* __restrict__ w4,
                                                  const float* __restrict__ b4, const double* __restrict__ c,
                                                  double* __restrict__ c_out, float* __restrict__ o_out, int H, int W,
                                                  NetParams P, double* __restrict__ part) {
    __shared__ __align__(16) uint8_t rows[3 * ROW_B];
    __shared__ float ws[9 * 32];
    __shared__ double red[2][NT / 32];
    const uint32_t rows_a = tc::smem_u32(rows);
    for (int i = threadIdx.x; i < 9 * 32; i += NT) ws[i] = w4[i];
    const int b = blockIdx.y;
    const int tpr = W / TILE, ntile = H * tpr;
    const int per = (ntile + gridDim.x - 1) / gridDim.x;
    const int t0 = blockIdx.x * per, t1 = min(t0 + per, ntile);
    const float bias = b4[0];
    double sc = 0.0, so = 0.0;
    int have = -1000000, seg_have = -1;  // row resident in slot (row % 3) up to `have`
    for (int t = t0; t < t1; ++t) {
        const int seg = t / H, y = t - seg * H, x0 = seg * TILE;
        __syncthreads();  // previous tile done with the rows about to be replaced
        const bool cont = seg == seg_have && y == have;  // rows y-2 .. y resident: stage only y+1
        for (int r = cont ? 2 : 0; r < 3; ++r)
            stage_row_async<NT>(rows_a, ((y - 1 + r) % 3 + 3) % 3, h3, b, y - 1 + r, x0, H, W);
        cp_async_commit();
        cp_async_wait_all();
        have = y + 1;
        seg_have = seg;
        __syncthreads();
        float s = 0.f;
#pragma unroll
        for (int ky = 0; ky < 3; ++ky) {
            const int slot = ((y - 1 + ky) % 3 + 3) % 3;
#pragma unroll
            for (int kx = 0; kx < 3; ++kx) {
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    float f[8];
                    unpack8(*reinterpret_cast<const uint4*>(rows + slot * ROW_B + k * CHUNK_B + (threadIdx.x + kx) * 16),
                            f);
#pragma unroll
                    for (int e = 0; e < 8; ++e) s = fmaf(f[e], ws[(ky * 3 + kx) * 32 + 8 * k + e], s);
                }
            }
        }
        const size_t p = ((size_t)b * H + y) * W + x0 + threadIdx.x;
        const float o = s + bias;
        if (o_out) o_out[p] = o;
        if (c_out) {
            const double cv = c[p], co = cv + P.out_scale * (double)o;
            c_out[p] = co;
            sc += cv;
            so += co;
        }
    }
    if (!c_out) return;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sc += __shfl_xor_sync(0xffffffffu, sc, o);
        so += __shfl_xor_sync(0xffffffffu, so, o);
    }
    if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = sc; red[1][threadIdx.x >> 5] = so; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a0 = 0.0, a1 = 0.0;
        for (int w = 0; w < NT / 32; ++w) { a0 += red[0][w]; a1 += red[1][w]; }
        part[((size_t)b * gridDim.x + blockIdx.x) * 2 + 0] = a0;
        part[((size_t)b * gridDim.x + blockIdx.x) * 2 + 1] = a1;
    }
}

// Mass correction per image from layer4_rows' partials: one warp per image,
// lane l sums partials l, l+32, ... (8 independent accumulators, then a fixed
// combination and a fixed shuffle tree, so the result is deterministic).
__global__ void __launch_bounds__(32) mass_correction(const double* __restrict__ part, int nparts, size_t npix,
                                                      double* __restrict__ corr) {
    const int img = blockIdx.x;
    double sa[8] = {0, 0, 0, 0, 0, 0, 0, 0}, sb[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const double* pp = part + (size_t)img * nparts * 2;
    for (int k0 = threadIdx.x; k0 < nparts; k0 += 32 * 8) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int k = k0 + 32 * q;
            if (k < nparts) {
                sa[q] += pp[2 * k];
                sb[q] += pp[2 * k + 1];
            }
        }
    }
    double a = 0.0, b = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        a += sa[q];
        b += sb[q];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if (threadIdx.x == 0) corr[img] = (a - b) / (double)npix;
}

// c_out += corr[image]: the mean-mass projection.
__global__ void __launch_bounds__(256) apply_correction(double* __restrict__ c_out, const double* __restrict__ corr,
                                                        size_t npix) {
    const int img = blockIdx.y;
    const double cr = corr[img];
    for (size_t p = blockIdx.x * 256ull + threadIdx.x; p < npix; p += (size_t)gridDim.x * 256)
        c_out[img * npix + p] += cr;
}

// ---------------------------------------------------------------------------
// One surrogate step in one kernel (inference)
// ---------------------------------------------------------------------------
// Each CTA takes a window of FW output pixels of one image and a strip of
// output rows, and streams the strip's rows through the four layers, all on
// the tensor cores: layer 1 as one UMMA (M128 N32 K16) over a 9-tap im2col
// tile, layers 2 and 3 as 18 UMMAs (M128 N32 K16), layer 4 as 18 UMMAs
// (M128 N16 K16, output channel 0 of 16; the other 15 weight rows are zero).
// The CUDA cores build the im2col tiles and run the epilogues.
//
// Ticks.  At tick t three warps issue this tick's UMMAs into TMEM accumulator
// set t & 1 (one thread per accumulator chain) while 16 warps run the
// epilogues of tick t - 1's UMMAs (set (t - 1) & 1), so the tensor cores and
// the epilogues overlap:
//   tick t UMMAs:      layer 1 -> row Y-4+t, layer 2 -> Y-7+t,
//                      layer 3 -> Y-10+t, layer 4 -> Y-13+t;
//   tick t epilogues:  the rows of tick t - 1;  im2col of row Y-3+t.
// A layer reads rows whose epilogues ran by the previous tick, so a strip of
// R output rows takes R + 14 ticks.  Activations live in rings of 5 staged
// rows ([8-channel chunk][130 px][8], as conv32_rows_tc's input rows): a row
// is read by the UMMAs of the three ticks after its epilogue, and the last of
// those completes before the epilogue that reuses its slot.
//
// Window pixels: a window with first output pixel X computes layer 1 on
// x = X-3 .. X+124, layer 2 on X-2 .., layer 3 on X-1 .., and keeps layer 4
// on X .. X+FW-1 (each 128-wide UMMA row loses one valid pixel at each side
// per layer).  c_out = c + out_scale * o is written without the mass
// projection; each CTA's FP64 sums of c and c_out go to part[job] and
// finish_projection applies the correction.
constexpr int FW = 122;                      // output pixels per window
constexpr int F_EW = 16;                     // epilogue warps: TMEM lane quadrant (w % 4), 8-channel chunk (w / 4)
constexpr int F_NT = 32 * (F_EW + 3);        // + three warps that issue the UMMAs (layers 1-2, 3, 4)
constexpr int IM_B = 2 * TILE * 16;          // 4096: im2col tile [k chunk][128 px][8] bf16 (taps 0-7 | 8, 0..)
constexpr int W1PK_B = 2 * 32 * 16;          // 1024: layer-1 weights [k chunk][32 n][8]
constexpr int W4PK_B = 9 * 2 * 2 * 16 * 16;  // 9216: layer-4 weights [tap][k16][chunk][16 n][8]
constexpr int F_RING = 5, F_IMS = 3;
constexpr int F_H1 = 0, F_H2 = F_H1 + F_RING * ROW_B, F_H3 = F_H2 + F_RING * ROW_B, F_IM = F_H3 + F_RING * ROW_B,
              F_W2 = F_IM + F_IMS * IM_B, F_W3 = F_W2 + WPK_B, F_W1 = F_W3 + WPK_B, F_W4 = F_W1 + W1PK_B,
              F_BAR = F_W4 + W4PK_B, F_SMEM = F_BAR + 128;
static_assert(F_SMEM <= 227 * 1024, "fused step exceeds shared memory");

// GELU (tanh form) of two values on the packed f32x2 instructions:
// 0.5 x (1 + tanh(k (x + c x^3))), with h = 0.5 x and y = fma(h, t, h).
__device__ __forceinline__ float2 gelu2(float2 x) {
    const float2 x2 = __fmul2_rn(x, x);
    const float2 in = __ffma2_rn(__fmul2_rn(make_float2(0.044715f, 0.044715f), x2), x, x);
    const float2 u = __fmul2_rn(make_float2(0.7978845608028654f, 0.7978845608028654f), in);
    const float2 t = make_float2(tanh_hw(u.x), tanh_hw(u.y));
    const float2 h = __fmul2_rn(make_float2(0.5f, 0.5f), x);
    return __ffma2_rn(h, t, h);
}

struct FusedArgs {
    const double* c;
    double* c_out;
    const __nv_bfloat16* wpk;   // layer-2 forward pack, then layer 3's (9216 elements each)
    const __nv_bfloat16* thin;  // layer-1 pack (512 elements), then layer 4's (4608)
    const float *b1, *b2, *b3, *b4;
    double* part;               // [job][2]: sums of c and c_out over the job's output pixels
    int* err;
    int H, W, nwin, nstrip, rows;
    NetParams P;
};

__device__ __forceinline__ int fring(int q) { return (q % F_RING + F_RING) % F_RING; }

__global__ void __launch_bounds__(F_NT, 1) step_fused_tc(const FusedArgs a) {
    extern __shared__ __align__(1024) uint8_t sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + F_BAR);  // [layer][set]
    uint32_t* slot_t = reinterpret_cast<uint32_t*>(sm + F_BAR + 64);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int job = blockIdx.x;
    const int b = job / (a.nwin * a.nstrip), rem = job - b * a.nwin * a.nstrip;
    const int win = rem / a.nstrip, strip = rem - win * a.nstrip;
    const int X = win * FW, Y = strip * a.rows, R = min(a.rows, a.H - Y);

    // weights in, rings and im2col tiles zeroed (the two pixels past each
    // 128-pixel row are read by the UMMAs but never written)
    {
        const uint4* w = reinterpret_cast<const uint4*>(a.wpk);
        uint4* d = reinterpret_cast<uint4*>(sm + F_W2);
        for (int u = threadIdx.x; u < 2 * WPK_B / 16; u += F_NT) d[u] = __ldg(w + u);
        const uint4* th = reinterpret_cast<const uint4*>(a.thin);
        uint4* dt = reinterpret_cast<uint4*>(sm + F_W1);
        for (int u = threadIdx.x; u < (W1PK_B + W4PK_B) / 16; u += F_NT) dt[u] = __ldg(th + u);
        uint4* z = reinterpret_cast<uint4*>(sm);
        for (int u = threadIdx.x; u < F_W2 / 16; u += F_NT) z[u] = make_uint4(0u, 0u, 0u, 0u);
    }
    if (warp == 0) {
        tc::tmem_alloc(slot_t, 256);
        tc::tmem_relinquish();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 8; ++k) tc::mbar_init(bar + k, 1);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *slot_t;
    const uint32_t id32 = tc::idesc_bf16_f32(128, 32, 0, 0), id16 = tc::idesc_bf16_f32(128, 16, 0, 0);
    const uint32_t sa = tc::smem_u32(sm);
    const uint64_t w1d = tc::sdesc(sa + F_W1, 512, 128), w2d = tc::sdesc(sa + F_W2, 512, 128),
                   w3d = tc::sdesc(sa + F_W3, 512, 128), w4d = tc::sdesc(sa + F_W4, 256, 128);
    const int quad = warp & 3, chunk = warp >> 2;
    const bool ew = warp < F_EW;  // an epilogue warp
    float2 bias1[4], bias2[4], bias3[4];
    const int bc = ew ? 8 * chunk : 0;  // the issue warp loads (and never uses) chunk 0's
#pragma unroll
    for (int n = 0; n < 4; ++n) {
        bias1[n] = make_float2(__ldg(a.b1 + bc + 2 * n), __ldg(a.b1 + bc + 2 * n + 1));
        bias2[n] = make_float2(__ldg(a.b2 + bc + 2 * n), __ldg(a.b2 + bc + 2 * n + 1));
        bias3[n] = make_float2(__ldg(a.b3 + bc + 2 * n), __ldg(a.b3 + bc + 2 * n + 1));
    }
    const float b4 = __ldg(a.b4);
    uint32_t phase[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
    uint32_t pending = 0u;  // barriers with a commit not yet waited for (thread 0's copy, which waits on all, is used)
    bool failed = false;
    double sc = 0.0, so = 0.0;

    // rows of tick t: layer 1, 2, 3, 4 and whether each is in its range
    auto row_of = [&](int k, int t) { return Y - (k == 0 ? 4 : k == 1 ? 7 : k == 2 ? 10 : 13) + t; };
    auto live = [&](int k, int t) {
        return k == 0 ? (t >= 1 && t < R + 7) : k == 1 ? (t >= 5 && t < R + 9) : k == 2 ? (t >= 9 && t < R + 11)
                                                                                      : (t >= 13 && t < R + 13);
    };
    // GELU epilogue of a 32-channel accumulator (TMEM column col) into the
    // staged row of ring `off` for row r: pixel quad*32 + lane, channels
    // 8*chunk .. 8*chunk + 7
    auto act_row = [&](uint32_t col, const float2* bias, int off, int r) {
        float v[8];
        tc::tmem_ld8(tmem + ((uint32_t)(quad * 32) << 16) + col + (uint32_t)(8 * chunk), v);
        uint32_t pk[4];
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            const float2 g = gelu2(__fadd2_rn(make_float2(v[2 * n], v[2 * n + 1]), bias[n]));
            pk[n] = pack2(g.x, g.y);
        }
        *reinterpret_cast<uint4*>(sm + off + fring(r) * ROW_B + chunk * CHUNK_B + (quad * 32 + lane) * 16) =
            make_uint4(pk[0], pk[1], pk[2], pk[3]);
    };
    // warp-uniform, so that a warp either runs its tcgen05.ld whole or not at all
    auto wait = [&](int k) {
        const bool ok = __all_sync(0xffffffffu, tc::mbar_wait_bounded(bar + k, phase[k], WAIT_NS));
        if (!ok) {
            failed = true;
            return false;
        }
        phase[k] ^= 1u;
        pending &= ~(1u << k);
        tc::fence_after_sync();
        return true;
    };

    const int nticks = R + 14;
    for (int t = 0; t < nticks; ++t) {
        const int set = t & 1;
        const uint32_t tset = tmem + (uint32_t)(128 * set);
        if (warp >= F_EW && lane == 0) {
            // Shared-memory descriptors are linear in the address (bits 0-13 =
            // address / 16, no carry below 256 KB), so each UMMA's descriptors
            // are a per-row base plus a compile-time offset.  One thread per
            // accumulator chain issues (layers 1-2, layer 3, layer 4), each
            // committing its own barriers: a single issuing thread is bound by
            // the issue latency of its UMMAs.
            const int iw = warp - F_EW;
            if (iw == 0 && live(0, t)) {
                const uint64_t ad = tc::sdesc(sa + F_IM + ((t - 1) % F_IMS) * IM_B, TILE * 16, 128);
                tc::umma_bf16(tset, ad, w1d, id32, 0);
                tc::umma_commit(bar + 0 * 2 + set);
            }
            auto conv = [&](int in_off, uint64_t wd, int r, uint32_t col, uint32_t id, int wblk) {
                uint64_t rd[3];
#pragma unroll
                for (int ky = 0; ky < 3; ++ky) rd[ky] = tc::sdesc(sa + in_off + fring(r - 1 + ky) * ROW_B, CHUNK_B, 128);
#pragma unroll
                for (int tap = 0; tap < 9; ++tap)
#pragma unroll
                    for (int kk = 0; kk < 2; ++kk) {
                        const int ky = tap / 3, kx = tap % 3;
                        const uint64_t ad = rd[ky] + (uint64_t)((2 * kk * CHUNK_B + kx * 16) >> 4);
                        const uint64_t bd = wd + (uint64_t)(((tap * 2 + kk) * wblk) >> 4);
                        tc::umma_bf16(tset + col, ad, bd, id, (tap | kk) != 0);
                    }
            };
            if (iw == 0 && live(1, t)) { conv(F_H1, w2d, row_of(1, t), 32, id32, 1024); tc::umma_commit(bar + 1 * 2 + set); }
            if (iw == 1 && live(2, t)) { conv(F_H2, w3d, row_of(2, t), 64, id32, 1024); tc::umma_commit(bar + 2 * 2 + set); }
            if (iw == 2 && live(3, t)) { conv(F_H3, w4d, row_of(3, t), 96, id16, 512); tc::umma_commit(bar + 3 * 2 + set); }
        }
        for (int k = 0; k < 4; ++k)
            if (live(k, t)) pending |= 1u << (2 * k + set);
        // im2col of layer-1 row Y-3+t for the next tick (pixel m <-> x = X-3+m):
        // the c values are loaded now and stored after the epilogues
        const bool im = ew && t < R + 6 && threadIdx.x < TILE;
        double cv9[9];
        if (im) {
            const int m = threadIdx.x, ry = Y - 3 + t, x = X - 3 + m;
#pragma unroll
            for (int k = 0; k < 9; ++k)
                cv9[k] = __ldg(a.c + ((size_t)b * a.H + wrap(ry - 1 + k / 3, a.H)) * a.W + wrap(x - 1 + k % 3, a.W));
        }
        // epilogues of the previous tick's UMMAs
        const int e = t - 1, es = e & 1;
        const uint32_t eset = (uint32_t)(128 * es);
        if (ew && e >= 0) {
            if (live(0, e) && !failed && wait(0 * 2 + es)) act_row(eset + 0, bias1, F_H1, row_of(0, e));
            if (live(1, e) && !failed && wait(1 * 2 + es)) act_row(eset + 32, bias2, F_H2, row_of(1, e));
            if (live(2, e) && !failed && wait(2 * 2 + es)) act_row(eset + 64, bias3, F_H3, row_of(2, e));
            if (live(3, e) && !failed && wait(3 * 2 + es) && chunk == 0) {
                float v[8];
                tc::tmem_ld8(tmem + ((uint32_t)(quad * 32) << 16) + eset + 96u, v);
                const int m = quad * 32 + lane, x = X + m;
                if (m < FW && x < a.W) {
                    const size_t p = ((size_t)b * a.H + row_of(3, e)) * a.W + x;
                    const float o = v[0] + b4;
                    const double cv = __ldg(a.c + p), co = cv + a.P.out_scale * (double)o;
                    a.c_out[p] = co;
                    sc += cv;
                    so += co;
                }
            }
        }
        if (im) {  // x0 = bf16((c - in_shift) * in_scale), as layer1_fwd's x0_at
            float v[9];
#pragma unroll
            for (int k = 0; k < 9; ++k)
                v[k] = __bfloat162float(__float2bfloat16_rn((float)((cv9[k] - a.P.in_shift) * a.P.in_scale)));
            uint8_t* dst = sm + F_IM + (t % F_IMS) * IM_B + threadIdx.x * 16;
            *reinterpret_cast<uint4*>(dst) =
                make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
            *reinterpret_cast<uint4*>(dst + TILE * 16) = make_uint4(pack2(v[8], 0.f), 0u, 0u, 0u);
        }
        // generic-proxy ring writes -> the next tick's UMMAs
        tc::fence_async_smem();
        tc::fence_before_sync();
        if (__syncthreads_or(failed)) {
            failed = true;
            break;
        }
        tc::fence_after_sync();
    }
    // a failed CTA may leave UMMAs in flight: wait (bounded) for the last
    // commit of each barrier before the TMEM is released
    if (failed && threadIdx.x == 0)
        for (int k = 0; k < 8; ++k)
            if (pending & (1u << k)) tc::mbar_wait_bounded(bar + k, phase[k], WAIT_NS);

    __shared__ double red[2][F_NT / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sc += __shfl_xor_sync(0xffffffffu, sc, o);
        so += __shfl_xor_sync(0xffffffffu, so, o);
    }
    if (lane == 0) { red[0][warp] = sc; red[1][warp] = so; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0;
        for (int w = 0; w < F_NT / 32; ++w) { s0 += red[0][w]; s1 += red[1][w]; }
        a.part[2 * job] = s0;
        a.part[2 * job + 1] = s1;
        if (failed) atomicExch(a.err, 1);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 256);
}

// The mean-mass projection after step_fused_tc: every block sums its image's
// job partials in the same fixed order, then adds the correction to its
// share of the image's pixels.
__global__ void __launch_bounds__(256) finish_projection(double* __restrict__ c_out, const double* __restrict__ part,
                                                         int jobs_per_img, size_t npix) {
    const int img = blockIdx.y;
    __shared__ double corr_s;
    if (threadIdx.x < 32) {
        double s0 = 0.0, s1 = 0.0;
        for (int j = threadIdx.x; j < jobs_per_img; j += 32) {
            s0 += part[2 * ((size_t)img * jobs_per_img + j)];
            s1 += part[2 * ((size_t)img * jobs_per_img + j) + 1];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s0 += __shfl_xor_sync(0xffffffffu, s0, o);
            s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        }
        if (threadIdx.x == 0) corr_s = (s0 - s1) / (double)npix;
    }
    __syncthreads();
    const double cr = corr_s;
    for (size_t p = blockIdx.x * 256ull + threadIdx.x; p < npix; p += (size_t)gridDim.x * 256)
        c_out[img * npix + p] += cr;
}

// Layer-1 and layer-4 operands of step_fused_tc (bf16):
//   thin[0 .. 511]      [k chunk][32 n][8]              = W1[n][8 chunk + e] (taps 9..15: 0)
//   thin[512 .. 5119]   [tap][k16][chunk][16 n][8]      = W4[tap][16 k16 + 8 chunk + e] for n = 0, else 0
__global__ void pack_thin(const float* __restrict__ W1, const float* __restrict__ W4, __nv_bfloat16* __restrict__ thin) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 512) {
        const int e = i % 8, n = (i / 8) % 32, kc = i / 256, k = 8 * kc + e;
        thin[i] = __float2bfloat16_rn(k < 9 ? W1[n * 9 + k] : 0.f);
    } else if (i < 512 + 4608) {
        const int r = i - 512;
        const int e = r % 8, n = (r / 8) % 16, chunk = (r / 128) % 2, kk = (r / 256) % 2, tap = r / 512;
        thin[i] = __float2bfloat16_rn(n == 0 ? W4[tap * 32 + 16 * kk + 8 * chunk + e] : 0.f);
    }
}

// Per-image FP64 sums of a and b (grid-stride per image: one block row per image).
__global__ void __launch_bounds__(256) image_sums(const double* __restrict__ a, const double* __restrict__ bb,
                                                  size_t npix, double* __restrict__ out) {
    const int img = blockIdx.y;
    double sa = 0.0, sb = 0.0;
    for (size_t p = blockIdx.x * 256ull + threadIdx.x; p < npix; p += (size_t)gridDim.x * 256) {
        sa += a[img * npix + p];
        sb += bb[img * npix + p];
    }
    __shared__ double sh[2][8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sa += __shfl_xor_sync(0xffffffffu, sa, o);
        sb += __shfl_xor_sync(0xffffffffu, sb, o);
    }
    if ((threadIdx.x & 31) == 0) { sh[0][threadIdx.x >> 5] = sa; sh[1][threadIdx.x >> 5] = sb; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ta = 0.0, tb = 0.0;
        for (int w = 0; w < 8; ++w) { ta += sh[0][w]; tb += sh[1][w]; }
        out[2 * ((size_t)img * gridDim.x + blockIdx.x) + 0] = ta;
        out[2 * ((size_t)img * gridDim.x + blockIdx.x) + 1] = tb;
    }
}

// c_out += (sum(c) - sum(c_out)) / npix per image: the mean-mass projection.
__global__ void __launch_bounds__(256) project_mass(double* __restrict__ c_out, const double* __restrict__ sums,
                                                    int nparts, size_t npix) {
    const int img = blockIdx.y;
    double sa = 0.0, sb = 0.0;
    for (int k = 0; k < nparts; ++k) {
        sa += sums[2 * ((size_t)img * nparts + k)];
        sb += sums[2 * ((size_t)img * nparts + k) + 1];
    }
    const double corr = (sa - sb) / (double)npix;
    for (size_t p = blockIdx.x * 256ull + threadIdx.x; p < npix; p += (size_t)gridDim.x * 256)
        c_out[img * npix + p] += corr;
}

// ---------------------------------------------------------------------------
// training kernels (CUDA cores)
// ---------------------------------------------------------------------------
// do = 2 (o - t) / N with t = (c_next - c) / out_scale; loss partials per block.
__global__ void __launch_bounds__(256) loss_grad(const float* __restrict__ o, const double* __restrict__ c,
                                                 const double* __restrict__ cn, float* __restrict__ dO, size_t N,
                                                 NetParams P, double* __restrict__ lpart) {
    double s = 0.0;
    for (size_t p = blockIdx.x * 256ull + threadIdx.x; p < N; p += (size_t)gridDim.x * 256) {
        const double t = (cn[p] - c[p]) / P.out_scale;
        const double d = (double)o[p] - t;
        dO[p] = (float)(2.0 * d / (double)N);
        s += d * d;
    }
    __shared__ double sh[8];
#pragma unroll
    for (int k = 16; k > 0; k >>= 1) s += __shfl_xor_sync(0xffffffffu, s, k);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += sh[w];
        lpart[blockIdx.x] = t;
    }
}

// Layer 4 backward: dz3[p][ci] = (sum_tap dO[p - tap] w4[tap][ci]) * gelu'(z3[p][ci]).
__global__ void __launch_bounds__(256) layer4_dgrad(const float* __restrict__ dO, const float* __restrict__ w4,
                                                    const __nv_bfloat16* __restrict__ z3, __nv_bfloat16* __restrict__ dz3,
                                                    int B, int H, int W) {
    __shared__ float ws[9 * 32];
    for (int i = threadIdx.x; i < 9 * 32; i += 256) ws[i] = w4[i];
    __syncthreads();
    const size_t N = (size_t)B * H * W;
    for (size_t p = blockIdx.x * 256ull + threadIdx.x; p < N; p += (size_t)gridDim.x * 256) {
        const int b = (int)(p / ((size_t)H * W)), y = (int)((p / W) % H), x = (int)(p % W);
        float d[9];
#pragma unroll
        for (int t = 0; t < 9; ++t)
            d[t] = dO[((size_t)b * H + wrap(y - (t / 3 - 1), H)) * W + wrap(x - (t % 3 - 1), W)];
        const uint4* zp = reinterpret_cast<const uint4*>(z3 + p * CH);
        uint4* out = reinterpret_cast<uint4*>(dz3 + p * CH);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float zf[8], g[8];
            unpack8(__ldg(zp + q), zf);
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                float s = 0.f;
#pragma unroll
                for (int t = 0; t < 9; ++t) s = fmaf(d[t], ws[t * 32 + 8 * q + e], s);
                g[e] = s * gelu_grad_f(zf[e]);
            }
            out[q] = make_uint4(pack2(g[0], g[1]), pack2(g[2], g[3]), pack2(g[4], g[5]), pack2(g[6], g[7]));
        }
    }
}

// Weight gradient of a thin layer on CUDA cores, one partial per block:
//   mode 4: dw4[tap][ci] = sum_p dO[p] h3[p + tap][ci],  db4 = sum_p dO[p]
//   mode 1: dw1[n][tap]  = sum_p dz1[p][n] x0[p + tap], db1[n] = sum_p dz1[p][n]
// Thread j < 288 owns one weight; threads 288..319 own bias terms.
// The block walks row segments of TILE pixels.
__global__ void __launch_bounds__(320) thin_wgrad(int mode, const float* __restrict__ dO,
                                                  const __nv_bfloat16* __restrict__ act, const double* __restrict__ c,
                                                  int B, int H, int W, NetParams P, float* __restrict__ partial) {
    __shared__ float dsh[TILE * 32];      // mode 4: dO of the segment; mode 1: dz1[px][n]
    __shared__ float xsh[3][TILE + 2][1];  // mode 1: x0 rows
    const int j = threadIdx.x;
    float acc = 0.f;
    const int tpr = W / TILE;
    const int ntiles = B * H * tpr;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int b = t / (H * tpr), rem = t - b * H * tpr, y = rem / tpr, x0 = (rem - y * tpr) * TILE;
        const size_t base = ((size_t)b * H + y) * W + x0;
        __syncthreads();
        if (mode == 4) {
            for (int i = j; i < TILE; i += 320) dsh[i] = dO[base + i];
        } else {
            for (int i = j; i < TILE * 32; i += 320) dsh[i] = __bfloat162float(act[(base + i / 32) * CH + i % 32]);
            for (int i = j; i < 3 * (TILE + 2); i += 320) {
                const int r = i / (TILE + 2), k = i % (TILE + 2);
                xsh[r][k][0] = x0_at(c, b, wrap(y + r - 1, H), wrap(x0 - 1 + k, W), H, W, P);
            }
        }
        __syncthreads();
        if (mode == 4) {
            if (j < 288) {
                const int tap = j / 32, ci = j % 32, ky = tap / 3 - 1, kx = tap % 3 - 1;
                const size_t row = ((size_t)b * H + wrap(y + ky, H)) * W;
                for (int i = 0; i < TILE; ++i)
                    acc = fmaf(dsh[i], __bfloat162float(act[(row + wrap(x0 + i + kx, W)) * CH + ci]), acc);
            } else if (j == 288) {
                for (int i = 0; i < TILE; ++i) acc += dsh[i];
            }
        } else {
            if (j < 288) {
                const int n = j / 9, tap = j % 9, ky = tap / 3, kx = tap % 3;
                for (int i = 0; i < TILE; ++i) acc = fmaf(dsh[i * 32 + n], xsh[ky][i + kx][0], acc);
            } else {
                const int n = j - 288;
                for (int i = 0; i < TILE; ++i) acc += dsh[i * 32 + n];
            }
        }
    }
    partial[(size_t)blockIdx.x * 320 + j] = acc;
}

// Column sums of dz [N][32] -> per-block partial [32] (bias gradient).
__global__ void __launch_bounds__(256) bias_grad(const __nv_bfloat16* __restrict__ dz, size_t N,
                                                 float* __restrict__ partial) {
    __shared__ float sh[8][32];
    const int c = threadIdx.x & 31, r = threadIdx.x >> 5;
    float s = 0.f;
    for (size_t p = blockIdx.x * 8ull + r; p < N; p += (size_t)gridDim.x * 8) s += __bfloat162float(dz[p * CH + c]);
    sh[r][c] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        float t = 0.f;
        for (int k = 0; k < 8; ++k) t += sh[k][threadIdx.x];
        partial[(size_t)blockIdx.x * 32 + threadIdx.x] = t;
    }
}

// Adam on the flat FP32 parameter vector (bias-corrected).
__global__ void adam_step(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// Rebuild the BF16 operands from the FP32 master parameters:
//   layers 2, 3 forward pack  [tap][k16][chunk][n][8]       = W[n][tap][16k16 + 8chunk + e]
//   layers 2, 3 dgrad pack    [tap'][k16][chunk][ci][8]     = W[16k16 + 8chunk + e][8 - tap'][ci]
//   layer 1 / 4 bf16-rounded float copies.
__global__ void pack_weights(const float* __restrict__ W2, const float* __restrict__ W3, const float* __restrict__ W1,
                             const float* __restrict__ W4, __nv_bfloat16* __restrict__ pk, float* __restrict__ w1r,
                             float* __restrict__ w4r) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    constexpr int P = 9 * 2 * 2 * 32 * 8;  // 9216 elements per pack
    if (i < 4 * P) {
        const int which = i / P, r = i % P;
        const int e = r % 8, row = (r / 8) % 32, chunk = (r / 256) % 2, kk = (r / 512) % 2, tap = r / 1024;
        const float* Wl = (which & 1) ? W3 : W2;
        float v;
        if (which < 2) {  // forward: row = n, k = (tap, ci)
            const int ci = 16 * kk + 8 * chunk + e;
            v = Wl[((size_t)row * 9 + tap) * 32 + ci];
        } else {          // dgrad: row = ci, k = (tap', n)
            const int n = 16 * kk + 8 * chunk + e;
            v = Wl[((size_t)n * 9 + (8 - tap)) * 32 + row];
        }
        pk[i] = __float2bfloat16_rn(v);
    } else if (i < 4 * P + 288) {
        const int k = i - 4 * P;
        w1r[k] = __bfloat162float(__float2bfloat16_rn(W1[k]));
    } else if (i < 4 * P + 576) {
        const int k = i - 4 * P - 288;
        w4r[k] = __bfloat162float(__float2bfloat16_rn(W4[k]));
    }
}

// Extract the compact [H][W] FP64 plane of a 2-D stored field (ghost g).
__global__ void gather_plane(const double* __restrict__ stored, double* __restrict__ out, int H, int W, int g) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    const int sx = W + 2 * g, sy = H + 2 * g;
    out[(size_t)y * W + x] = stored[(size_t)g * sx * sy + (size_t)(y + g) * sx + (x + g)];
}
__global__ void scatter_plane(const double* __restrict__ in, double* __restrict__ stored, int H, int W, int g) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    const int sx = W + 2 * g, sy = H + 2 * g;
    stored[(size_t)g * sx * sy + (size_t)(y + g) * sx + (x + g)] = in[(size_t)y * W + x];
}

}  // namespace sg
}  // namespace phix

using namespace phix;
using namespace phix::sg;

// Parameter vector layout (FP32): W1[32][9] b1[32] W2[32][9][32] b2[32] W3[32][9][32] b3[32] W4[9][32] b4[1]
// with W[n][ky][kx][ci] flattened (ky, kx) -> tap.
namespace {
constexpr int OFF_W1 = 0, OFF_B1 = 288, OFF_W2 = 320, OFF_B2 = 320 + 9216, OFF_W3 = OFF_B2 + 32,
              OFF_B3 = OFF_W3 + 9216, OFF_W4 = OFF_B3 + 32, OFF_B4 = OFF_W4 + 288, NPARAM = OFF_B4 + 1;
}

struct phix_surrogate {
    int H = 0, W = 0, bmax = 0, nsm = 148;
    NetParams P{};
    float* params = nullptr;  // NPARAM master FP32
    float* grads = nullptr;
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    int adam_t = 0;
    __nv_bfloat16* pk = nullptr;  // 4 packs
    float* w1r = nullptr;
    float* w4r = nullptr;
    __nv_bfloat16 *z1 = nullptr, *h1 = nullptr, *z2 = nullptr, *h2 = nullptr, *z3 = nullptr, *h3 = nullptr;
    __nv_bfloat16 *dz = nullptr, *dz2 = nullptr;  // gradient scratch
    float* o = nullptr;
    float* dO = nullptr;
    double* sums = nullptr;
    float* partial = nullptr;  // weight-gradient partials
    float* thin_out = nullptr; // reduced gradients of the thin layers (320)
    double* lpart = nullptr;
    int* err = nullptr;
    bool packed = false;
    __nv_bfloat16* thin = nullptr;  // layer-1 and layer-4 UMMA operands of the fused step
    bool fused = true;              // phix_surrogate_step: one fused kernel (else the layer kernels)
};

namespace {

int sg_conv_grid(const phix_surrogate* s, int B) {
    const int ntiles = B * s->H * (s->W / TILE);
    const int g = s->nsm * 4;
    return ntiles < g ? ntiles : g;
}

int sg_pack(phix_surrogate* s, cudaStream_t st) {
    const int total = 4 * 9216 + 576;
    pack_weights<<<(total + 255) / 256, 256, 0, st>>>(s->params + OFF_W2, s->params + OFF_W3, s->params + OFF_W1,
                                                      s->params + OFF_W4, s->pk, s->w1r, s->w4r);
    PHIX_LAUNCH_CHECK("pack_weights");
    pack_thin<<<(512 + 4608 + 255) / 256, 256, 0, st>>>(s->params + OFF_W1, s->params + OFF_W4, s->thin);
    PHIX_LAUNCH_CHECK("pack_thin");
    s->packed = true;
    return PHIX_OK;
}

constexpr size_t ROWS_SMEM = WPK_B + RING * ROW_B + 2 * 8 + 8;

int sg_conv_rows(phix_surrogate* s, const ConvArgs& a, cudaStream_t st) {
    const int tpr = a.W / TILE;
    const long long tiles = (long long)a.B * a.H * tpr;
    const int slots = s->nsm * 3;  // 3 CTAs of ~60 KB shared memory per SM
    int rows = (int)((tiles + slots - 1) / slots);
    if (rows < 2) rows = 2;
    const long long jobs = (long long)a.B * tpr * ((a.H + rows - 1) / rows);
    const int grid = (int)(jobs < slots ? jobs : slots);
    conv32_rows_tc<<<grid, NT_ROWS, ROWS_SMEM, st>>>(a, rows);
    PHIX_LAUNCH_CHECK("conv32_rows_tc");
    return PHIX_OK;
}

// One surrogate step as step_fused_tc + finish_projection: strips of
// ceil(B * windows * H / SMs) rows, so the jobs fill one wave of one CTA per SM.
int sg_step_fused(phix_surrogate* s, const double* c, int B, double* c_out, cudaStream_t st) {
    FusedArgs a{};
    a.c = c; a.c_out = c_out; a.wpk = s->pk; a.thin = s->thin;
    a.b1 = s->params + OFF_B1; a.b2 = s->params + OFF_B2; a.b3 = s->params + OFF_B3; a.b4 = s->params + OFF_B4;
    a.part = s->sums; a.err = s->err;
    a.H = s->H; a.W = s->W; a.P = s->P;
    a.nwin = (s->W + FW - 1) / FW;
    const long long rows_total = (long long)B * a.nwin * s->H;
    a.rows = (int)((rows_total + s->nsm - 1) / s->nsm);
    if (a.rows < 1) a.rows = 1;
    a.nstrip = (s->H + a.rows - 1) / a.rows;
    const int jobs_per_img = a.nwin * a.nstrip, njobs = B * jobs_per_img;
    step_fused_tc<<<njobs, F_NT, F_SMEM, st>>>(a);
    PHIX_LAUNCH_CHECK("step_fused_tc");
    const size_t npix = (size_t)s->H * s->W;
    int pb = (int)((npix + 255) / 256);
    const int pmax = (s->nsm * 4 + B - 1) / B;
    pb = pb < pmax ? pb : pmax;
    finish_projection<<<dim3(pb, B), 256, 0, st>>>(c_out, s->sums, jobs_per_img, npix);
    PHIX_LAUNCH_CHECK("finish_projection");
    return PHIX_OK;
}

int sg_forward(phix_surrogate* s, const double* c, int B, double* c_out, float* o_out, cudaStream_t st,
               bool keep_z = true) {
    int rc;
    if (!s->packed && (rc = sg_pack(s, st))) return rc;
    if (s->fused && c_out && !o_out && !keep_z) return sg_step_fused(s, c, B, c_out, st);
    const size_t N = (size_t)B * s->H * s->W;
    const int eg = (int)((N + 255) / 256 < (size_t)s->nsm * 8 ? (N + 255) / 256 : (size_t)s->nsm * 8);
    layer1_fwd<<<eg, 256, 0, st>>>(c, s->w1r, s->params + OFF_B1, keep_z ? s->z1 : nullptr, s->h1, B, s->H, s->W,
                                   s->P);
    PHIX_LAUNCH_CHECK("layer1_fwd");
    ConvArgs a{};
    a.B = B; a.H = s->H; a.W = s->W; a.err = s->err;
    a.x = s->h1; a.wpk = s->pk; a.bias = s->params + OFF_B2; a.out = s->h2; a.zout = keep_z ? s->z2 : nullptr;
    if ((rc = sg_conv_rows(s, a, st))) return rc;
    a.x = s->h2; a.wpk = s->pk + 9216; a.bias = s->params + OFF_B3; a.out = s->h3; a.zout = keep_z ? s->z3 : nullptr;
    if ((rc = sg_conv_rows(s, a, st))) return rc;
    const int tiles = s->H * (s->W / TILE);
    int nb = (tiles + 1) / 2;  // two segments (consecutive rows) per block
    nb = nb < L4_MAXBLK ? nb : L4_MAXBLK;
    layer4_rows<<<dim3(nb, B), NT, 0, st>>>(s->h3, s->w4r, s->params + OFF_B4, c, c_out, o_out, s->H, s->W, s->P,
                                            s->sums);
    PHIX_LAUNCH_CHECK("layer4_rows");
    if (c_out) {
        const size_t npix = (size_t)s->H * s->W;
        int pb = (int)((npix + 255) / 256);
        const int pmax = (s->nsm * 4 + B - 1) / B;
        pb = pb < pmax ? pb : pmax;
        double* corr = s->sums + (size_t)2 * L4_MAXBLK * s->bmax;
        mass_correction<<<B, 32, 0, st>>>(s->sums, nb, npix, corr);
        PHIX_LAUNCH_CHECK("mass_correction");
        apply_correction<<<dim3(pb, B), 256, 0, st>>>(c_out, corr, npix);
        PHIX_LAUNCH_CHECK("apply_correction");
    }
    return PHIX_OK;
}

}  // namespace

extern "C" {

int phix_surrogate_create(phix_surrogate_t** out, int H, int W, int batch_max, double in_shift, double in_scale,
                          double out_scale) {
    if (!out || H < 3 || W < TILE || W % TILE != 0 || batch_max < 1) {
        set_error("surrogate_create: need H >= 3, W a multiple of %d, batch_max >= 1", TILE);
        return PHIX_ERR_ARG;
    }
    *out = nullptr;
    auto* s = new (std::nothrow) phix_surrogate();
    if (!s) { set_error("out of host memory"); return PHIX_ERR_ARG; }
    s->H = H; s->W = W; s->bmax = batch_max;
    {
        cudaError_t ea = cudaFuncSetAttribute(conv32_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, WGRAD_SMEM);
        if (ea != cudaSuccess) { delete s; return cuda_status(ea, "cudaFuncSetAttribute(wgrad)"); }
        ea = cudaFuncSetAttribute(conv32_rows_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ROWS_SMEM);
        if (ea != cudaSuccess) { delete s; return cuda_status(ea, "cudaFuncSetAttribute(conv rows)"); }
        ea = cudaFuncSetAttribute(step_fused_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, F_SMEM);
        if (ea != cudaSuccess) { delete s; return cuda_status(ea, "cudaFuncSetAttribute(fused step)"); }
    }
    s->P.in_shift = in_shift; s->P.in_scale = in_scale; s->P.out_scale = out_scale;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&s->nsm, cudaDevAttrMultiProcessorCount, dev);
    const size_t N = (size_t)batch_max * H * W;
    const int cgmax = s->nsm * 4;
    cudaError_t e = cudaSuccess;
    auto A = [&](void** p, size_t bytes) { if (e == cudaSuccess) e = cudaMalloc(p, bytes); };
    A((void**)&s->params, NPARAM * 4); A((void**)&s->grads, NPARAM * 4);
    A((void**)&s->adam_m, NPARAM * 4); A((void**)&s->adam_v, NPARAM * 4);
    A((void**)&s->pk, 4 * 9216 * 2); A((void**)&s->w1r, 288 * 4); A((void**)&s->w4r, 288 * 4);
    A((void**)&s->thin, (512 + 4608) * 2);
    for (auto** p : {&s->z1, &s->h1, &s->z2, &s->h2, &s->z3, &s->h3, &s->dz, &s->dz2}) A((void**)p, N * CH * 2);
    A((void**)&s->o, N * 4); A((void**)&s->dO, N * 4);
    A((void**)&s->sums, sizeof(double) * (2 * L4_MAXBLK + 1) * batch_max);  // partials + corrections
    A((void**)&s->partial, sizeof(float) * (size_t)cgmax * 9216 + sizeof(float) * 320 * cgmax);
    A((void**)&s->lpart, sizeof(double) * s->nsm * 8);
    A((void**)&s->thin_out, sizeof(float) * 320);
    A((void**)&s->err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(s->err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(s->params, 0, NPARAM * 4);
    if (e == cudaSuccess) e = cudaMemset(s->adam_m, 0, NPARAM * 4);
    if (e == cudaSuccess) e = cudaMemset(s->adam_v, 0, NPARAM * 4);
    if (e != cudaSuccess) {
        int rc = cuda_status(e, "surrogate_create");
        phix_surrogate_destroy(s);
        return rc;
    }
    *out = s;
    return PHIX_OK;
}

int phix_surrogate_destroy(phix_surrogate_t* s) {
    if (!s) return PHIX_OK;
    for (void* p : {(void*)s->params, (void*)s->grads, (void*)s->adam_m, (void*)s->adam_v, (void*)s->pk,
                    (void*)s->w1r, (void*)s->w4r, (void*)s->z1, (void*)s->h1, (void*)s->z2, (void*)s->h2,
                    (void*)s->z3, (void*)s->h3, (void*)s->dz, (void*)s->dz2, (void*)s->o, (void*)s->dO,
                    (void*)s->sums, (void*)s->partial, (void*)s->lpart, (void*)s->err, (void*)s->thin_out,
                    (void*)s->thin})
        if (p) cudaFree(p);
    delete s;
    return PHIX_OK;
}

int phix_surrogate_nparams(void) { return NPARAM; }

int phix_surrogate_set_fused(phix_surrogate_t* s, int on) {
    if (!s) { set_error("surrogate_set_fused: NULL surrogate"); return PHIX_ERR_ARG; }
    s->fused = on != 0;
    return PHIX_OK;
}

int phix_surrogate_set_params(phix_surrogate_t* s, const float* host_params) {
    if (!s || !host_params) { set_error("set_params: NULL"); return PHIX_ERR_ARG; }
    PHIX_TRY_CUDA(cudaMemcpy(s->params, host_params, NPARAM * 4, cudaMemcpyHostToDevice));
    s->packed = false;
    s->adam_t = 0;
    PHIX_TRY_CUDA(cudaMemset(s->adam_m, 0, NPARAM * 4));
    PHIX_TRY_CUDA(cudaMemset(s->adam_v, 0, NPARAM * 4));
    return PHIX_OK;
}

int phix_surrogate_get_params(phix_surrogate_t* s, float* host_params, float* host_grads) {
    if (!s) { set_error("get_params: NULL"); return PHIX_ERR_ARG; }
    if (host_params) PHIX_TRY_CUDA(cudaMemcpy(host_params, s->params, NPARAM * 4, cudaMemcpyDeviceToHost));
    if (host_grads) PHIX_TRY_CUDA(cudaMemcpy(host_grads, s->grads, NPARAM * 4, cudaMemcpyDeviceToHost));
    return PHIX_OK;
}

// c_out = projection(c + out_scale * net(c)); c, c_out: [B][H][W] FP64 device.
int phix_surrogate_step(phix_surrogate_t* s, const double* c, double* c_out, int B, void* stream) {
    if (!s || !c || !c_out || B < 1 || B > s->bmax) { set_error("surrogate_step: bad argument"); return PHIX_ERR_ARG; }
    return sg_forward(s, c, B, c_out, nullptr, (cudaStream_t)stream, false);
}

// Network output o (no update) for tests: o [B][H][W] FP32 device; also leaves
// the activations of this batch in the internal buffers.
int phix_surrogate_forward(phix_surrogate_t* s, const double* c, float* o, int B, void* stream) {
    if (!s || !c || !o || B < 1 || B > s->bmax) { set_error("surrogate_forward: bad argument"); return PHIX_ERR_ARG; }
    return sg_forward(s, c, B, nullptr, o, (cudaStream_t)stream);
}

// Gradients of the MSE loss mean((o - (c_next - c)/out_scale)^2) into the
// internal gradient vector; *loss receives the loss (synchronous).
int phix_surrogate_grad(phix_surrogate_t* s, const double* c, const double* c_next, int B, double* loss,
                        void* stream) {
    if (!s || !c || !c_next || B < 1 || B > s->bmax) { set_error("surrogate_grad: bad argument"); return PHIX_ERR_ARG; }
    cudaStream_t st = (cudaStream_t)stream;
    int rc = sg_forward(s, c, B, nullptr, s->o, st);
    if (rc) return rc;
    const size_t N = (size_t)B * s->H * s->W;
    const int eg = (int)((N + 255) / 256 < (size_t)s->nsm * 8 ? (N + 255) / 256 : (size_t)s->nsm * 8);
    loss_grad<<<eg, 256, 0, st>>>(s->o, c, c_next, s->dO, N, s->P, s->lpart);
    PHIX_LAUNCH_CHECK("loss_grad");
    const int cg = sg_conv_grid(s, B);
    // The weight-gradient CTAs hold 128 TMEM columns each; asking for 56 KiB
    // of shared memory keeps at most 4 of them on an SM (512 columns).
    const size_t smem_c = WPK_B + 3 * ROW_B + 16, smem_w = WGRAD_SMEM;
    float* part_w = s->partial;                      // cg x 9216
    float* part_t = s->partial + (size_t)cg * 9216;  // cg x 320
    // layer 4
    thin_wgrad<<<cg, 320, 0, st>>>(4, s->dO, s->h3, c, B, s->H, s->W, s->P, part_t);
    PHIX_LAUNCH_CHECK("thin_wgrad(4)");
    float* t4 = s->thin_out;  // 288 weights, then the bias at 288
    reduce_partials<<<2, 256, 0, st>>>(part_t, cg, 320, t4);
    PHIX_LAUNCH_CHECK("reduce_partials");
    PHIX_TRY_CUDA(cudaMemcpyAsync(s->grads + OFF_W4, t4, 288 * 4, cudaMemcpyDeviceToDevice, st));
    PHIX_TRY_CUDA(cudaMemcpyAsync(s->grads + OFF_B4, t4 + 288, 4, cudaMemcpyDeviceToDevice, st));
    layer4_dgrad<<<eg, 256, 0, st>>>(s->dO, s->w4r, s->z3, s->dz, B, s->H, s->W);
    PHIX_LAUNCH_CHECK("layer4_dgrad");
    // layers 3 and 2: weight gradient, bias gradient, data gradient
    const __nv_bfloat16* acts_in[2] = {s->h2, s->h1};
    const __nv_bfloat16* zprev[2] = {s->z2, s->z1};
    const int offW[2] = {OFF_W3, OFF_W2}, offB[2] = {OFF_B3, OFF_B2};
    const __nv_bfloat16* dpk[2] = {s->pk + 3 * 9216, s->pk + 2 * 9216};
    __nv_bfloat16* dz_in = s->dz;
    __nv_bfloat16* dz_out = s->dz2;
    for (int l = 0; l < 2; ++l) {
        WgradArgs w{};
        w.x = acts_in[l]; w.dz = dz_in; w.partial = part_w; w.B = B; w.H = s->H; w.W = s->W; w.err = s->err;
        conv32_wgrad_tc<<<cg, NT, smem_w, st>>>(w);
        PHIX_LAUNCH_CHECK("conv32_wgrad_tc");
        reduce_partials<<<(9216 + 255) / 256, 256, 0, st>>>(part_w, cg, 9216, s->grads + offW[l]);
        PHIX_LAUNCH_CHECK("reduce_partials");
        bias_grad<<<cg, 256, 0, st>>>(dz_in, N, part_t);
        PHIX_LAUNCH_CHECK("bias_grad");
        reduce_partials<<<1, 32, 0, st>>>(part_t, cg, 32, s->grads + offB[l]);
        PHIX_LAUNCH_CHECK("reduce_partials");
        ConvArgs a{};
        a.B = B; a.H = s->H; a.W = s->W; a.err = s->err;
        a.x = dz_in; a.wpk = dpk[l]; a.zaux = zprev[l]; a.out = dz_out;
        conv32_tc<EPI_DGRAD><<<cg, NT, smem_c, st>>>(a);
        PHIX_LAUNCH_CHECK("conv32_tc<dgrad>");
        __nv_bfloat16* tmp = dz_in;
        dz_in = dz_out;
        dz_out = tmp;
    }
    // layer 1 (dz_in now holds dz1)
    thin_wgrad<<<cg, 320, 0, st>>>(1, nullptr, dz_in, c, B, s->H, s->W, s->P, part_t);
    PHIX_LAUNCH_CHECK("thin_wgrad(1)");
    reduce_partials<<<2, 256, 0, st>>>(part_t, cg, 320, t4);
    PHIX_LAUNCH_CHECK("reduce_partials");
    PHIX_TRY_CUDA(cudaMemcpyAsync(s->grads + OFF_W1, t4, 288 * 4, cudaMemcpyDeviceToDevice, st));
    PHIX_TRY_CUDA(cudaMemcpyAsync(s->grads + OFF_B1, t4 + 288, 32 * 4, cudaMemcpyDeviceToDevice, st));
    // loss
    std::vector<double> lp(eg);
    PHIX_TRY_CUDA(cudaMemcpyAsync(lp.data(), s->lpart, sizeof(double) * eg, cudaMemcpyDeviceToHost, st));
    int herr = 0;
    PHIX_TRY_CUDA(cudaMemcpyAsync(&herr, s->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    PHIX_TRY_CUDA(cudaStreamSynchronize(st));
    if (herr) { set_error("surrogate: a tensor-core wait timed out"); return PHIX_ERR_TIMEOUT; }
    double tot = 0.0;
    for (double v : lp) tot += v;
    if (loss) *loss = tot / (double)N;
    return PHIX_OK;
}

// Adam update of the master parameters with the current gradient vector, then
// repack the BF16 operands.  `grads` (device, may be null) replaces the
// internal gradient vector first (data-parallel training passes the averaged
// gradients here).
int phix_surrogate_adam(phix_surrogate_t* s, const float* grads, float lr, void* stream) {
    if (!s) { set_error("adam: NULL"); return PHIX_ERR_ARG; }
    cudaStream_t st = (cudaStream_t)stream;
    if (grads) PHIX_TRY_CUDA(cudaMemcpyAsync(s->grads, grads, NPARAM * 4, cudaMemcpyDeviceToDevice, st));
    s->adam_t += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)s->adam_t), c2 = 1.f - powf(b2, (float)s->adam_t);
    adam_step<<<(NPARAM + 255) / 256, 256, 0, st>>>(s->params, s->grads, s->adam_m, s->adam_v, NPARAM, lr, b1, b2,
                                                    1e-8f, c1, c2);
    PHIX_LAUNCH_CHECK("adam_step");
    return sg_pack(s, st);
}

// Reads and clears the surrogate's device error flag (set by a kernel whose
// bounded tensor-core wait gave up); synchronous on `stream`.
int phix_surrogate_status(phix_surrogate_t* s, void* stream) {
    if (!s) { set_error("surrogate_status: NULL surrogate"); return PHIX_ERR_ARG; }
    cudaStream_t st = (cudaStream_t)stream;
    int herr = 0;
    PHIX_TRY_CUDA(cudaMemcpyAsync(&herr, s->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    PHIX_TRY_CUDA(cudaMemsetAsync(s->err, 0, sizeof(int), st));
    PHIX_TRY_CUDA(cudaStreamSynchronize(st));
    if (herr) { set_error("surrogate: a tensor-core wait timed out"); return PHIX_ERR_TIMEOUT; }
    return PHIX_OK;
}

// Device pointer of the internal FP32 gradient vector (NPARAM floats).
float* phix_surrogate_grad_ptr(phix_surrogate_t* s) { return s ? s->grads : nullptr; }

// Compact [H][W] plane <-> 2-D stored FP64 field with ghost g.
int phix_plane_gather(const double* stored, double* plane, int H, int W, int ghost, void* stream) {
    if (!stored || !plane || H < 1 || W < 1 || ghost < 0) { set_error("plane_gather: bad argument"); return PHIX_ERR_ARG; }
    gather_plane<<<dim3((W + 255) / 256, H), 256, 0, (cudaStream_t)stream>>>(stored, plane, H, W, ghost);
    PHIX_LAUNCH_CHECK("gather_plane");
    return PHIX_OK;
}
int phix_plane_scatter(const double* plane, double* stored, int H, int W, int ghost, void* stream) {
    if (!stored || !plane || H < 1 || W < 1 || ghost < 0) { set_error("plane_scatter: bad argument"); return PHIX_ERR_ARG; }
    scatter_plane<<<dim3((W + 255) / 256, H), 256, 0, (cudaStream_t)stream>>>(plane, stored, H, W, ghost);
    PHIX_LAUNCH_CHECK("scatter_plane");
    return PHIX_OK;
}

// Self-test of the bounded mbarrier wait of the tensor-core kernels: one
// thread initialises a barrier of count 1, arrives on it when `arrive`, and
// waits for its first phase with a wall-clock limit.  With no arrival the wait
// gives up after limit_ns and the kernel records that in the flag and
// returns, as the tensor-core kernels do, leaving the context usable.
__global__ void wait_selftest(int arrive, unsigned long long limit_ns, int* flag) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0) return;
    tc::mbar_init(&bar, 1);
    if (arrive) tc::mbar_arrive(&bar);
    if (!tc::mbar_wait_bounded(&bar, 0, limit_ns)) atomicExch(flag, 1);
}

static __device__ int g_wait_selftest_flag;

int phix_wait_selftest(int arrive, double limit_s, void* stream) {
    if (!(limit_s > 0.0 && limit_s <= 2.0)) { set_error("wait_selftest: limit %g s outside (0, 2]", limit_s); return PHIX_ERR_ARG; }
    cudaStream_t st = (cudaStream_t)stream;
    const int zero = 0;
    PHIX_TRY_CUDA(cudaMemcpyToSymbolAsync(g_wait_selftest_flag, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, st));
    int* flag = nullptr;  // device address of the flag (the symbol is a host-side stand-in)
    PHIX_TRY_CUDA(cudaGetSymbolAddress((void**)&flag, g_wait_selftest_flag));
    wait_selftest<<<1, 32, 0, st>>>(arrive, (unsigned long long)(limit_s * 1e9), flag);
    PHIX_LAUNCH_CHECK("wait_selftest");
    int herr = 0;
    PHIX_TRY_CUDA(cudaMemcpyFromSymbolAsync(&herr, g_wait_selftest_flag, sizeof(int), 0, cudaMemcpyDeviceToHost, st));
    PHIX_TRY_CUDA(cudaStreamSynchronize(st));
    if (herr) { set_error("wait_selftest: the bounded wait gave up after %g s", limit_s); return PHIX_ERR_TIMEOUT; }
    return PHIX_OK;
}

}  // extern "C"
