// noalloc.cu -- mass / free-energy diagnostics that allocate no memory.
//
// phix_reduce_mass_energy obtains its scratch (per-block partial sums) with
// cudaMallocAsync on every call.  Some callers cannot allocate device memory:
// hosts whose device memory is owned and pre-reserved by another runtime or a
// custom allocator (an allocation from this library would fail or break that
// owner's accounting), and embedded or real-time loops that forbid allocation
// after start-up.  phix_reduce_mass_energy_noalloc gives them the same
// diagnostics with the scratch in a file-scope device array instead.
//
// The call is synchronous: it copies the result to the host and waits for
// `stream`.  So it must not be made on a stream under capture, and with
// stream = NULL (the legacy default stream) no global-mode capture may be
// active in the process.
//
// Scratch: one (mass, energy, non-finite count) triple per physical row of
// the grid (n[1] * n[2] rows) plus the three result slots, in
// g_noalloc_rows[3 * PHIX_NOALLOC_MAX_ROWS + 3] (about 1.5 MiB).  Every GPU
// that loads the library holds this array until the process exits.  Each call
// overwrites every slot it reads, so nothing needs clearing between calls,
// but all calls share the one array: calls that overlap on the GPU (on
// different streams, or from different host threads) race and must be
// serialised by the caller.
//
// The array's device address is looked up once per device (the first call
// there) and kept for the life of the process.  It belongs to that device's
// primary context: a process that destroys the context (cudaDeviceReset) must
// not call this entry point on that device afterwards.
#include <cmath>
#include <mutex>

#include "phix/detail/common.cuh"
#include "stepper.h"

namespace phix {
namespace {

constexpr int NA_WARPS = 8;

static __device__ __align__(256) double g_noalloc_rows[3 * PHIX_NOALLOC_MAX_ROWS + 3];

// Device address of g_noalloc_rows on each device (host code must not use
// the symbol itself: on the host it is only a stand-in).
constexpr int NA_MAX_DEVICES = 64;
double* g_rows_addr[NA_MAX_DEVICES] = {nullptr};
std::mutex g_rows_mu;

int rows_address(double** out) {
    int dev = 0;
    PHIX_TRY_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NA_MAX_DEVICES) { set_error("noalloc: device index %d out of range", dev); return PHIX_ERR_ARG; }
    std::lock_guard<std::mutex> lock(g_rows_mu);
    if (!g_rows_addr[dev]) {
        double* p = nullptr;
        PHIX_TRY_CUDA(cudaGetSymbolAddress((void**)&p, g_noalloc_rows));
        g_rows_addr[dev] = p;
    }
    *out = g_rows_addr[dev];
    return PHIX_OK;
}

struct NaParams {
    Layout L;
    int dim, phys, nf;
    double kap[2];
    double prm[5];
    double inv2d[3];
    double dv;
};

__device__ __forceinline__ double na_mapped(const double* u, const Layout& L, int dim, int px, int py, int pz) {
    int q[3] = {px, py, pz}, p[3] = {px, py, pz};
    double cval;
    for (int a = 0; a < dim; ++a)
        if (map_axis(p[a], L.n[a], L.bc[2 * a], L.bc[2 * a + 1], L.bcv[2 * a], L.bcv[2 * a + 1], L.ghost, &q[a],
                     &cval) == MAP_CONST)
            return cval;
    return u[L.origin + q[0] + L.s[1] * q[1] + L.s[2] * q[2]];
}

// One warp per physical row (j, k): the row's sums go to rows[3 * row + {0,1,2}].
__global__ void __launch_bounds__(32 * NA_WARPS) na_rows(const double* __restrict__ u0, const double* __restrict__ u1,
                                                         NaParams P, double* __restrict__ rows, int nrows) {
    const int row = blockIdx.x * NA_WARPS + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (row >= nrows) return;
    const int j = row % P.L.n[1], k = row / P.L.n[1];
    double m = 0.0, e = 0.0, bad = 0.0;
    for (int i = lane; i < P.L.n[0]; i += 32) {
        const int idx = P.L.origin + i + P.L.s[1] * j + P.L.s[2] * k;
        const double x = u0[idx];
        const double y = P.nf > 1 ? u1[idx] : 0.0;
        if (!isfinite(x) || !isfinite(y)) bad += 1.0;
        double fb;
        if (P.phys == PHIX_PHYS_AC) {
            fb = 0.25 * (x * x - 1.0) * (x * x - 1.0);
        } else if (P.phys == PHIX_PHYS_CH) {
            fb = P.prm[2] * (x - P.prm[3]) * (x - P.prm[3]) * (P.prm[4] - x) * (P.prm[4] - x);
        } else {
            fb = x * x * (1.0 - x) * (1.0 - x) + y * y * (1.0 - y) * (1.0 - y) + P.prm[4] * x * x * y * y;
        }
        double gr = 0.0;
        for (int f = 0; f < P.nf; ++f) {
            const double* u = f == 0 ? u0 : u1;
            double g2 = 0.0;
            for (int a = 0; a < P.dim; ++a) {
                int dp[3] = {i, j, k}, dm[3] = {i, j, k};
                dp[a] += 1;
                dm[a] -= 1;
                const double d = (na_mapped(u, P.L, P.dim, dp[0], dp[1], dp[2]) -
                                  na_mapped(u, P.L, P.dim, dm[0], dm[1], dm[2])) * P.inv2d[a];
                g2 += d * d;
            }
            gr += 0.5 * P.kap[f] * g2;
        }
        m += x;
        e += fb + gr;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m += __shfl_xor_sync(0xffffffffu, m, o);
        e += __shfl_xor_sync(0xffffffffu, e, o);
        bad += __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if (lane == 0) {
        rows[3 * row + 0] = m;
        rows[3 * row + 1] = e;
        rows[3 * row + 2] = bad;
    }
}

// One warp sums the row triples in a fixed order; result at rows[3 * nrows].
__global__ void __launch_bounds__(32) na_total(double* __restrict__ rows, int nrows, double dv) {
    double m = 0.0, e = 0.0, bad = 0.0;
    for (int r = threadIdx.x; r < nrows; r += 32) {
        m += rows[3 * r + 0];
        e += rows[3 * r + 1];
        bad += rows[3 * r + 2];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m += __shfl_xor_sync(0xffffffffu, m, o);
        e += __shfl_xor_sync(0xffffffffu, e, o);
        bad += __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if (threadIdx.x == 0) {
        rows[3 * nrows + 0] = m * dv;
        rows[3 * nrows + 1] = e * dv;
        rows[3 * nrows + 2] = bad;
    }
}

}  // namespace
}  // namespace phix

using namespace phix;

extern "C" int phix_reduce_mass_energy_noalloc(const double* const* fields, int phys, const double* prm,
                                               const phix_grid_t* g, double* out, void* stream) {
    if (!fields || !prm || !out || !g) { set_error("reduce_noalloc: NULL argument"); return PHIX_ERR_ARG; }
    const int nf = physics_nfields(phys);
    if (nf == 0) { set_error("reduce_noalloc: unknown physics %d", phys); return PHIX_ERR_ARG; }
    for (int f = 0; f < nf; ++f)
        if (!fields[f]) { set_error("reduce_noalloc: field %d NULL", f); return PHIX_ERR_ARG; }
    NaParams P{};
    int rc = validate_grid(g, &P.L, nullptr);
    if (rc) return rc;
    const long long nrows = (long long)g->n[1] * g->n[2];
    if (nrows > PHIX_NOALLOC_MAX_ROWS) {
        set_error("reduce_noalloc: grid has %lld rows (n[1]*n[2]); the allocation-free scratch holds at most %d",
                  nrows, PHIX_NOALLOC_MAX_ROWS);
        return PHIX_ERR_ARG;
    }
    double* rows = nullptr;
    if ((rc = rows_address(&rows))) return rc;
    P.dim = g->dim;
    P.phys = phys;
    P.nf = nf;
    for (int i = 0; i < 5; ++i) P.prm[i] = prm[i];
    if (phys == PHIX_PHYS_CHAC) { P.kap[0] = prm[2]; P.kap[1] = prm[3]; }
    else P.kap[0] = prm[1];
    P.dv = 1.0;
    for (int a = 0; a < 3; ++a) {
        P.inv2d[a] = a < g->dim ? 1.0 / (2.0 * g->d[a]) : 0.0;
        if (a < g->dim) P.dv *= g->d[a];
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int blocks = (int)((nrows + NA_WARPS - 1) / NA_WARPS);
    na_rows<<<blocks, 32 * NA_WARPS, 0, s>>>(fields[0], nf > 1 ? fields[1] : fields[0], P, rows, (int)nrows);
    PHIX_LAUNCH_CHECK("na_rows");
    na_total<<<1, 32, 0, s>>>(rows, (int)nrows, P.dv);
    PHIX_LAUNCH_CHECK("na_total");
    double res[3];
    PHIX_TRY_CUDA(cudaMemcpyAsync(res, rows + 3 * nrows, sizeof(res), cudaMemcpyDeviceToHost, s));
    PHIX_TRY_CUDA(cudaStreamSynchronize(s));
    out[0] = res[0];
    out[1] = res[1];
    if (res[2] != 0.0) { set_error("reduce_noalloc: %.0f non-finite cells", res[2]); return PHIX_ERR_NONFINITE; }
    return PHIX_OK;
}
