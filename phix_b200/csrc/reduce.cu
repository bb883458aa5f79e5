// reduce.cu -- FP64 mass and free-energy diagnostics (phix_reduce_mass_energy,
// phix_stepper_diagnostics).
//
//   mass   = sum_phys u * dV
//   energy = sum_phys [ f_bulk(u) + sum_fields kappa_f/2 |grad u_f|^2 ] * dV
// with central gradients on BC-mapped neighbours; with periodic BCs this is
// np.roll in develop/Spinodal Decomposition/computeFreeEnergy.py:76-98.
//
// Pass 1: grid-stride over physical cells, per-thread FP64 sums, warp-shuffle
// then shared-memory block reduction, one partial per block.  Pass 2: one
// block sums the partials in a fixed order.  The result is deterministic for a
// given grid.  Non-finite cells are counted, not trapped.
#include <cmath>

#include "phix/detail/common.cuh"
#include "stepper.h"

namespace phix {

namespace {

constexpr int RED_NT = 256;
constexpr int RED_MAX_BLOCKS = 148 * 8;

struct RedParams {
    Layout L;
    int dim, phys, nf;
    double kap[2];
    double prm[5];
    double inv2d[3];
    double dv;
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename T>
__device__ __forceinline__ double mapped(const T* u, const Layout& L, int dim, int px, int py, int pz) {
    int q[3] = {px, py, pz}, p[3] = {px, py, pz};
    double cval;
    for (int a = 0; a < dim; ++a)
        if (map_axis(p[a], L.n[a], L.bc[2 * a], L.bc[2 * a + 1], L.bcv[2 * a], L.bcv[2 * a + 1], L.ghost, &q[a],
                     &cval) == MAP_CONST)
            return cval;
    return (double)u[L.origin + q[0] + L.s[1] * q[1] + L.s[2] * q[2]];
}

template <typename T>
__global__ void __launch_bounds__(RED_NT) red_pass1(const T* __restrict__ u0, const T* __restrict__ u1, RedParams P,
                                                    double* __restrict__ partials) {
    const long long N = (long long)P.L.n[0] * P.L.n[1] * P.L.n[2];
    double m = 0.0, e = 0.0, bad = 0.0;
    for (long long c = blockIdx.x * (long long)RED_NT + threadIdx.x; c < N; c += (long long)gridDim.x * RED_NT) {
        const int i = (int)(c % P.L.n[0]);
        const int j = (int)((c / P.L.n[0]) % P.L.n[1]);
        const int k = (int)(c / ((long long)P.L.n[0] * P.L.n[1]));
        const int idx = P.L.origin + i + P.L.s[1] * j + P.L.s[2] * k;
        const double x = (double)u0[idx];
        const double y = P.nf > 1 ? (double)u1[idx] : 0.0;
        if (!isfinite(x) || !isfinite(y)) bad += 1.0;
        double fb;
        if (P.phys == PHIX_PHYS_AC) {
            fb = 0.25 * (x * x - 1.0) * (x * x - 1.0);
        } else if (P.phys == PHIX_PHYS_CH) {
            const double rho = P.prm[2], ca = P.prm[3], cb = P.prm[4];
            fb = rho * (x - ca) * (x - ca) * (cb - x) * (cb - x);
        } else {
            const double lam = P.prm[4];
            fb = x * x * (1.0 - x) * (1.0 - x) + y * y * (1.0 - y) * (1.0 - y) + lam * x * x * y * y;
        }
        double gr = 0.0;
        for (int f = 0; f < P.nf; ++f) {
            const T* u = f == 0 ? u0 : u1;
            double g2 = 0.0;
            for (int a = 0; a < P.dim; ++a) {
                int dp[3] = {i, j, k}, dm[3] = {i, j, k};
                dp[a] += 1;
                dm[a] -= 1;
                const double d = (mapped(u, P.L, P.dim, dp[0], dp[1], dp[2]) -
                                  mapped(u, P.L, P.dim, dm[0], dm[1], dm[2])) * P.inv2d[a];
                g2 += d * d;
            }
            gr += 0.5 * P.kap[f] * g2;
        }
        m += x;
        e += fb + gr;
    }
    __shared__ double sh[3][RED_NT / 32];
    m = warp_sum(m);
    e = warp_sum(e);
    bad = warp_sum(bad);
    const int w = threadIdx.x / 32, l = threadIdx.x % 32;
    if (l == 0) { sh[0][w] = m; sh[1][w] = e; sh[2][w] = bad; }
    __syncthreads();
    if (w == 0) {
        m = l < RED_NT / 32 ? sh[0][l] : 0.0;
        e = l < RED_NT / 32 ? sh[1][l] : 0.0;
        bad = l < RED_NT / 32 ? sh[2][l] : 0.0;
        m = warp_sum(m);
        e = warp_sum(e);
        bad = warp_sum(bad);
        if (l == 0) {
            partials[3 * blockIdx.x + 0] = m;
            partials[3 * blockIdx.x + 1] = e;
            partials[3 * blockIdx.x + 2] = bad;
        }
    }
}

__global__ void __launch_bounds__(32) red_pass2(double* __restrict__ partials, int nblocks, double dv) {
    double m = 0.0, e = 0.0, bad = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += 32) {
        m += partials[3 * b + 0];
        e += partials[3 * b + 1];
        bad += partials[3 * b + 2];
    }
    m = warp_sum(m);
    e = warp_sum(e);
    bad = warp_sum(bad);
    if (threadIdx.x == 0) {
        // result lands after the per-block partials
        partials[3 * nblocks + 0] = m * dv;
        partials[3 * nblocks + 1] = e * dv;
        partials[3 * nblocks + 2] = bad;
    }
}

int red_blocks(const phix_grid_t* g) {
    long long N = (long long)g->n[0] * g->n[1] * g->n[2];
    long long b = (N + RED_NT - 1) / RED_NT;
    return (int)(b < RED_MAX_BLOCKS ? (b > 0 ? b : 1) : RED_MAX_BLOCKS);
}

}  // namespace

int reduce_partials_needed(const phix_grid_t* g) { return 3 * red_blocks(g) + 3; }

template <typename T>
int reduce_mass_energy(const T* const* fields, int nf, int phys, const double* prm, const phix_grid_t* g,
                       double* partials, int partials_n, double* out, cudaStream_t s) {
    RedParams P{};
    int rc = validate_grid(g, &P.L, nullptr);
    if (rc) return rc;
    if (physics_nfields(phys) != nf) { set_error("diagnostics: physics %d needs %d fields", phys, physics_nfields(phys)); return PHIX_ERR_ARG; }
    P.dim = g->dim;
    P.phys = phys;
    P.nf = nf;
    for (int i = 0; i < 5; ++i) P.prm[i] = prm ? prm[i] : 0.0;
    if (phys == PHIX_PHYS_CHAC) { P.kap[0] = prm[2]; P.kap[1] = prm[3]; }
    else P.kap[0] = prm[1];
    P.dv = 1.0;
    for (int a = 0; a < 3; ++a) {
        P.inv2d[a] = a < g->dim ? 1.0 / (2.0 * g->d[a]) : 0.0;
        if (a < g->dim) P.dv *= g->d[a];
    }
    const int nb = red_blocks(g);
    if (partials_n < 3 * nb + 3) { set_error("diagnostics: partial buffer too small"); return PHIX_ERR_ARG; }
    red_pass1<T><<<nb, RED_NT, 0, s>>>(fields[0], nf > 1 ? fields[1] : fields[0], P, partials);
    PHIX_LAUNCH_CHECK("red_pass1");
    red_pass2<<<1, 32, 0, s>>>(partials, nb, P.dv);
    PHIX_LAUNCH_CHECK("red_pass2");
    double res[3];
    PHIX_TRY_CUDA(cudaMemcpyAsync(res, partials + 3 * nb, sizeof(res), cudaMemcpyDeviceToHost, s));
    PHIX_TRY_CUDA(cudaStreamSynchronize(s));
    out[0] = res[0];
    out[1] = res[1];
    if (res[2] != 0.0) { set_error("diagnostics: %.0f non-finite cells", res[2]); return PHIX_ERR_NONFINITE; }
    return PHIX_OK;
}
template int reduce_mass_energy<float>(const float* const*, int, int, const double*, const phix_grid_t*, double*, int,
                                       double*, cudaStream_t);
template int reduce_mass_energy<double>(const double* const*, int, int, const double*, const phix_grid_t*, double*,
                                        int, double*, cudaStream_t);

}  // namespace phix

using namespace phix;

extern "C" int phix_reduce_mass_energy(const double* const* fields, int phys, const double* prm, const phix_grid_t* g,
                                       double* out, void* stream) {
    if (!fields || !prm || !out || !g) { set_error("reduce: NULL argument"); return PHIX_ERR_ARG; }
    const int nf = physics_nfields(phys);
    if (nf == 0) { set_error("reduce: unknown physics %d", phys); return PHIX_ERR_ARG; }
    for (int f = 0; f < nf; ++f)
        if (!fields[f]) { set_error("reduce: field %d NULL", f); return PHIX_ERR_ARG; }
    int rc = validate_grid(g, nullptr, nullptr);
    if (rc) return rc;
    const int np = reduce_partials_needed(g);
    double* part = nullptr;
    PHIX_TRY_CUDA(cudaMallocAsync((void**)&part, sizeof(double) * np, (cudaStream_t)stream));
    rc = reduce_mass_energy<double>(fields, nf, phys, prm, g, part, np, out, (cudaStream_t)stream);
    cudaFreeAsync(part, (cudaStream_t)stream);
    return rc;
}
