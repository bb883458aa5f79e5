// ops.cu -- single-operator kernels for runtime-composed (unfused) right-hand
// sides: ghost refresh, Laplacian, gradient, pointwise and product accumulates,
// axpy.  Each replaces one of the reference's per-term kernels with the same
// arithmetic (rounding pinned as in stage.cuh) on a 2-D/3-D launch grid
// instead of the reference's 1-D grid with div/mod index recovery.
#include "phix/detail/common.cuh"
#include "stepper.h"

namespace phix {
namespace {

constexpr int OPS_TX = 32, OPS_TY = 8;

// physical-cell launch geometry: x by threads, y and z by grid
struct Cells {
    Layout L;
    int dim;
};

inline dim3 cell_grid(const Layout& L) {
    return dim3((L.n[0] + OPS_TX - 1) / OPS_TX, (L.n[1] + OPS_TY - 1) / OPS_TY, L.n[2]);
}

__device__ __forceinline__ bool cell_index(const Layout& L, int* idx) {
    const int i = blockIdx.x * OPS_TX + threadIdx.x, j = blockIdx.y * OPS_TY + threadIdx.y, k = blockIdx.z;
    if (i >= L.n[0] || j >= L.n[1]) return false;
    *idx = L.origin + i + L.s[1] * j + L.s[2] * k;
    return true;
}

template <int DIM>
__global__ void __launch_bounds__(OPS_TX* OPS_TY) k_lap(double* __restrict__ rhs, const double* __restrict__ src,
                                                        double coeff, Layout L, double i2x, double i2y, double i2z) {
    int c;
    if (!cell_index(L, &c)) return;
    const double f2 = rmul(2.0, src[c]);
    double tx = second_diff(src[c + 1], f2, src[c - 1]);
    double ty = DIM >= 2 ? second_diff(src[c + L.s[1]], f2, src[c - L.s[1]]) : 0.0;
    double tz = DIM >= 3 ? second_diff(src[c + L.s[2]], f2, src[c - L.s[2]]) : 0.0;
    rhs[c] = rfma(coeff, lap_combine<double, DIM>(tx, ty, tz, i2x, i2y, i2z), rhs[c]);
}

__global__ void __launch_bounds__(OPS_TX* OPS_TY) k_grad(double* __restrict__ rhs, const double* __restrict__ src,
                                                         double coeff, Layout L, int off, double inv2d) {
    int c;
    if (!cell_index(L, &c)) return;
    // rhs += coeff * (f[+] - f[-]) * inv_2d   (Equation.cu:123)
    rhs[c] = rfma(rmul(coeff, rsub(src[c + off], src[c - off])), inv2d, rhs[c]);
}

__global__ void __launch_bounds__(OPS_TX* OPS_TY) k_pw(double* __restrict__ rhs, const double* __restrict__ s1,
                                                       const double* __restrict__ s2, double coeff, int func, Layout L,
                                                       double two_rho, double ca, double cb, double two_lam) {
    int c;
    if (!cell_index(L, &c)) return;
    const double a = s1[c];
    double v;
    switch (func) {
        case PHIX_PW_IDENT: v = a; break;
        case PHIX_PW_AC: v = f_ac(a); break;
        case PHIX_PW_DW: v = f_dw(a, two_rho, ca, cb); break;
        case PHIX_PW_CHAC_C: v = f_chac_c(a, s2[c], two_lam); break;
        case PHIX_PW_CHAC_E: v = f_chac_e(a, s2[c], two_lam); break;
        default: v = rmul(a, s2[c]); break;  // PHIX_PW_MUL
    }
    rhs[c] = rfma(coeff, v, rhs[c]);  // TermPW.inl:36
}

__global__ void __launch_bounds__(OPS_TX* OPS_TY) k_mul(double* __restrict__ rhs, const double* __restrict__ s1,
                                                        const double* __restrict__ s2, double coeff, Layout L) {
    int c;
    if (!cell_index(L, &c)) return;
    rhs[c] = rfma(rmul(coeff, s1[c]), s2[c], rhs[c]);  // Equation.cu:403
}

__global__ void __launch_bounds__(256) k_axpy(double* __restrict__ dst, const double* __restrict__ src, double coeff,
                                              size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = rfma(coeff, src[i], dst[i]);
}

// One BC object's ghost fill over the full stored extent of the other two
// axes (ghost corners included, every layer), as in Boundary.cu:95-195.
// `low_part`: data is the low part of a compensated state (Dirichlet ghosts
// get 0, their value lives in the high part).
template <typename T>
__global__ void __launch_bounds__(256) k_bc_face(T* __restrict__ data, Layout L, int axis, int type, int do_lo,
                                                 int do_hi, double v_lo, double v_hi, int low_part) {
    if (low_part) v_lo = v_hi = 0.0;
    const int sx = L.s[1], sy = L.s[2] / L.s[1], sz = L.n[2] + 2 * L.ghost;
    int nf0, nf1, fs0, fs1, astr;
    if (axis == 0) { astr = 1; nf0 = sy; nf1 = sz; fs0 = sx; fs1 = sx * sy; }
    else if (axis == 1) { astr = sx; nf0 = sx; nf1 = sz; fs0 = 1; fs1 = sx * sy; }
    else { astr = sx * sy; nf0 = sx; nf1 = sy; fs0 = 1; fs1 = sx; }
    const int n = L.n[axis], g = L.ghost;
    const long long total = (long long)nf0 * nf1;
    for (long long t = blockIdx.x * 256LL + threadIdx.x; t < total; t += (long long)gridDim.x * 256) {
        const int t0 = (int)(t % nf0), t1 = (int)(t / nf0);
        const int off = t0 * fs0 + t1 * fs1;
        for (int l = 1; l <= g; ++l) {
            const int lo = (g - l) * astr + off, hi = (g + n + l - 1) * astr + off;
            if (type == PHIX_BC_PERIODIC) {
                data[lo] = data[(g + n - l) * astr + off];
                data[hi] = data[(g + l - 1) * astr + off];
            } else if (type == PHIX_BC_NOFLUX) {
                if (do_lo) data[lo] = data[g * astr + off];
                if (do_hi) data[hi] = data[(g + n - 1) * astr + off];
            } else {
                if (do_lo) data[lo] = (T)v_lo;
                if (do_hi) data[hi] = (T)v_hi;
            }
        }
    }
}

int check_ptrs(const void* a, const void* b = (const void*)1) {
    if (!a || !b) { set_error("NULL device pointer"); return PHIX_ERR_ARG; }
    return PHIX_OK;
}

void inv_d2(const phix_grid_t* g, double* i2) {
    for (int a = 0; a < 3; ++a) i2[a] = a < g->dim ? 1.0 / (g->d[a] * g->d[a]) : 0.0;
}

}  // namespace

// Every BC of the grid, in buildBCs order (BCFactory.cpp:50-74): axis x, y, z;
// a periodic axis is one BC object, otherwise the LOW then the HIGH side.
template <typename T>
int bc_fill(T* field, const phix_grid_t* g, bool low_part, cudaStream_t s) {
    Layout L;
    int rc = validate_grid(g, &L, nullptr);
    if (rc) return rc;
    return bc_fill_layout<T>(field, g, L, low_part, s);
}

// The same on an array of layout L (the grid's, or a stepper's row-padded
// internal copy: the padding columns past the x ghosts are never read).
template <typename T>
int bc_fill_layout(T* field, const phix_grid_t* g, const Layout& L, bool low_part, cudaStream_t s) {
    int rc;
    auto launch = [&](int axis, int type, int lo, int hi) -> int {
        const int sx = L.s[1], sy = L.s[2] / L.s[1], sz = L.n[2] + 2 * L.ghost;
        long long faces = axis == 0 ? (long long)sy * sz : axis == 1 ? (long long)sx * sz : (long long)sx * sy;
        int blocks = (int)((faces + 255) / 256);
        if (blocks > 148 * 8) blocks = 148 * 8;
        k_bc_face<T><<<blocks, 256, 0, s>>>(field, L, axis, type, lo, hi, g->bc_val[2 * axis], g->bc_val[2 * axis + 1],
                                            low_part ? 1 : 0);
        PHIX_LAUNCH_CHECK("k_bc_face");
        return PHIX_OK;
    };
    for (int a = 0; a < g->dim; ++a) {
        const int tl = g->bc_type[2 * a], th = g->bc_type[2 * a + 1];
        if (tl == PHIX_BC_PERIODIC) {
            if ((rc = launch(a, PHIX_BC_PERIODIC, 1, 1))) return rc;
            continue;
        }
        if (tl == PHIX_BC_NOFLUX || tl == PHIX_BC_FIXED)
            if ((rc = launch(a, tl, 1, 0))) return rc;
        if (th == PHIX_BC_NOFLUX || th == PHIX_BC_FIXED)
            if ((rc = launch(a, th, 0, 1))) return rc;
    }
    return PHIX_OK;
}
template int bc_fill<float>(float*, const phix_grid_t*, bool, cudaStream_t);
template int bc_fill<double>(double*, const phix_grid_t*, bool, cudaStream_t);
template int bc_fill_layout<float>(float*, const phix_grid_t*, const Layout&, bool, cudaStream_t);
template int bc_fill_layout<double>(double*, const phix_grid_t*, const Layout&, bool, cudaStream_t);

}  // namespace phix

using namespace phix;

extern "C" {

int phix_bc_apply(double* field, const phix_grid_t* g, void* stream) {
    int rc = validate_grid(g, nullptr, nullptr);
    if (rc || (rc = check_ptrs(field))) return rc;
    return bc_fill<double>(field, g, false, (cudaStream_t)stream);
}

int phix_lap_accumulate(double* rhs, const double* src, double coeff, const phix_grid_t* g, void* stream) {
    Layout L;
    int rc = validate_grid(g, &L, nullptr);
    if (rc || (rc = check_ptrs(rhs, src))) return rc;
    double i2[3];
    inv_d2(g, i2);
    dim3 blk(OPS_TX, OPS_TY);
    cudaStream_t s = (cudaStream_t)stream;
    if (g->dim == 1) k_lap<1><<<cell_grid(L), blk, 0, s>>>(rhs, src, coeff, L, i2[0], i2[1], i2[2]);
    else if (g->dim == 2) k_lap<2><<<cell_grid(L), blk, 0, s>>>(rhs, src, coeff, L, i2[0], i2[1], i2[2]);
    else k_lap<3><<<cell_grid(L), blk, 0, s>>>(rhs, src, coeff, L, i2[0], i2[1], i2[2]);
    PHIX_LAUNCH_CHECK("k_lap");
    return PHIX_OK;
}

int phix_grad_accumulate(double* rhs, const double* src, double coeff, int axis, const phix_grid_t* g,
                         void* stream) {
    Layout L;
    int rc = validate_grid(g, &L, nullptr);
    if (rc || (rc = check_ptrs(rhs, src))) return rc;
    if (axis < 0 || axis >= g->dim) { set_error("grad: axis out of range for this mesh dimension"); return PHIX_ERR_ARG; }
    k_grad<<<cell_grid(L), dim3(OPS_TX, OPS_TY), 0, (cudaStream_t)stream>>>(rhs, src, coeff, L, L.s[axis],
                                                                           0.5 / g->d[axis]);
    PHIX_LAUNCH_CHECK("k_grad");
    return PHIX_OK;
}

int phix_pointwise_accumulate(double* rhs, const double* s1, const double* s2, double coeff, int func,
                              const double* prm, const phix_grid_t* g, void* stream) {
    Layout L;
    int rc = validate_grid(g, &L, nullptr);
    if (rc || (rc = check_ptrs(rhs, s1))) return rc;
    if (func < PHIX_PW_IDENT || func > PHIX_PW_MUL) { set_error("pointwise: unknown functor %d", func); return PHIX_ERR_ARG; }
    const bool two = func == PHIX_PW_CHAC_C || func == PHIX_PW_CHAC_E || func == PHIX_PW_MUL;
    if (two && !s2) { set_error("pointwise: functor %d needs two fields", func); return PHIX_ERR_ARG; }
    const bool needs_prm = func == PHIX_PW_DW || func == PHIX_PW_CHAC_C || func == PHIX_PW_CHAC_E;
    if (needs_prm && !prm) { set_error("pointwise: functor %d needs prm", func); return PHIX_ERR_ARG; }
    double two_rho = 0, ca = 0, cb = 0, two_lam = 0;
    if (func == PHIX_PW_DW) { two_rho = 2.0 * prm[2]; ca = prm[3]; cb = prm[4]; }
    if (func == PHIX_PW_CHAC_C || func == PHIX_PW_CHAC_E) two_lam = 2.0 * prm[4];
    k_pw<<<cell_grid(L), dim3(OPS_TX, OPS_TY), 0, (cudaStream_t)stream>>>(rhs, s1, two ? s2 : s1, coeff, func, L,
                                                                         two_rho, ca, cb, two_lam);
    PHIX_LAUNCH_CHECK("k_pw");
    return PHIX_OK;
}

int phix_mul_accumulate(double* rhs, const double* s1, const double* s2, double coeff, const phix_grid_t* g,
                        void* stream) {
    Layout L;
    int rc = validate_grid(g, &L, nullptr);
    if (rc || (rc = check_ptrs(rhs, s1)) || (rc = check_ptrs(s2))) return rc;
    k_mul<<<cell_grid(L), dim3(OPS_TX, OPS_TY), 0, (cudaStream_t)stream>>>(rhs, s1, s2, coeff, L);
    PHIX_LAUNCH_CHECK("k_mul");
    return PHIX_OK;
}

int phix_axpy(double* dst, const double* src, double coeff, size_t n, void* stream) {
    int rc = check_ptrs(dst, src);
    if (rc) return rc;
    if (n == 0) return PHIX_OK;
    size_t blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_axpy<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(dst, src, coeff, n);
    PHIX_LAUNCH_CHECK("k_axpy");
    return PHIX_OK;
}

}  // extern "C"
