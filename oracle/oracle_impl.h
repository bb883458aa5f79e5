/*
 * oracle_impl.h -- body of the CPU oracle, instantiated twice by phix_oracle.c
 * (REAL = double -> *_f64, REAL = float -> *_f32).
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of PhiX's explicit
 * finite-difference time step, written to check the CUDA path.  Nothing in the
 * product links it; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it.
 *
 * It follows the reference algorithm structure literally: ghost-padded stored
 * arrays, BC kernels that fill whole ghost faces, one accumulate pass per DSL
 * term into a zeroed rhs, scratch materialisation for lap(expr, bcs), and the
 * GPU solver's RK4 stage semantics.  Citations are to the reference project.
 */

/* OpenMP build (liboracle_omp.so, -DOR_OMP): the per-cell loops and the
 * whole-array stage combinations run on all host threads.  Every cell's
 * arithmetic is unchanged, so both builds give the same bits. */
#ifndef OR_PAR
#ifdef OR_OMP
#define OR_PAR _Pragma("omp parallel for schedule(static)")
#define OR_PAR2 _Pragma("omp parallel for collapse(2) schedule(static)")
#else
#define OR_PAR
#define OR_PAR2
#endif
#endif

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SFX)

/* a*b + c, contracted (one rounding) in fma_mode 1, two roundings in mode 0.
 * Mode 0 reproduces the reference's x86-64 host build (no FMA contraction);
 * mode 1 reproduces the pattern nvcc's default -fmad=true gives the
 * reference's device kernels, and the pattern the sm_100a kernels pin with
 * __fma_rn. */
static inline REAL FN(madd)(int mode, REAL a, REAL b, REAL c) {
    if (mode) return FMA(a, b, c);
    volatile REAL p = a * b;   /* volatile: forbid contraction in mode 0 */
    return p + c;
}

/* ---------------------------------------------------------------------------
 * Boundary conditions.  Boundary.cu:95-195 (kernel_periodic / kernel_noflux /
 * kernel_fixed) with the face geometry of makeFaceParams (Boundary.cu:52-84):
 * one thread per position of the full stored extent of the two other axes,
 * ghost corners included, every ghost layer written.
 * ------------------------------------------------------------------------- */
static void FN(bc_face)(REAL* data, const or_grid_t* g, int axis, int type,
                        int do_low, int do_high, REAL value) {
    int sx = g->n[0] + 2 * g->ghost, sy = g->n[1] + 2 * g->ghost,
        sz = g->n[2] + 2 * g->ghost;
    int gh = g->ghost;
    int axis_stride, n_axis, nf0, nf1, fs0, fs1;
    if (axis == 0) { axis_stride = 1;       n_axis = g->n[0]; nf0 = sy; nf1 = sz; fs0 = sx; fs1 = sx * sy; }
    else if (axis == 1) { axis_stride = sx; n_axis = g->n[1]; nf0 = sx; nf1 = sz; fs0 = 1;  fs1 = sx * sy; }
    else { axis_stride = sx * sy;           n_axis = g->n[2]; nf0 = sx; nf1 = sy; fs0 = 1;  fs1 = sx; }
    OR_PAR
    for (int t0 = 0; t0 < nf0; ++t0)
        for (int t1 = 0; t1 < nf1; ++t1) {
            long off = (long)t0 * fs0 + (long)t1 * fs1;
            for (int l = 1; l <= gh; ++l) {
                long lo = (long)(gh - l) * axis_stride + off;
                long hi = (long)(gh + n_axis + l - 1) * axis_stride + off;
                if (type == OR_BC_PERIODIC) {
                    data[lo] = data[(long)(gh + n_axis - l) * axis_stride + off];
                    data[hi] = data[(long)(gh + l - 1) * axis_stride + off];
                } else if (type == OR_BC_NOFLUX) {
                    if (do_low) data[lo] = data[(long)gh * axis_stride + off];
                    if (do_high) data[hi] = data[(long)(gh + n_axis - 1) * axis_stride + off];
                } else if (type == OR_BC_FIXED) {
                    if (do_low) data[lo] = value;
                    if (do_high) data[hi] = value;
                }
            }
        }
}

/* Apply the BC list the way buildBCs orders it (BCFactory.cpp:50-74): axis x,
 * then y, then z; a periodic axis is one BC object, otherwise LOW then HIGH. */
void FN(or_bc_apply)(REAL* data, const or_grid_t* g) {
    for (int ax = 0; ax < g->dim; ++ax) {
        int tl = g->bc_type[2 * ax], th = g->bc_type[2 * ax + 1];
        if (tl == OR_BC_PERIODIC && th == OR_BC_PERIODIC) {
            FN(bc_face)(data, g, ax, OR_BC_PERIODIC, 1, 1, 0);
            continue;
        }
        if (tl == OR_BC_NOFLUX || tl == OR_BC_FIXED)
            FN(bc_face)(data, g, ax, tl, 1, 0, (REAL)g->bc_val[2 * ax]);
        if (th == OR_BC_NOFLUX || th == OR_BC_FIXED)
            FN(bc_face)(data, g, ax, th, 0, 1, (REAL)g->bc_val[2 * ax + 1]);
    }
}

/* ---------------------------------------------------------------------------
 * Stencil accumulates.  Equation.cu:40-80 (lap) and :89-124 (grad).
 * ------------------------------------------------------------------------- */
#define OR_LOOP_PHYS(g)                                                      \
    int sx = (g)->n[0] + 2 * (g)->ghost, sy = (g)->n[1] + 2 * (g)->ghost;    \
    int gh = (g)->ghost;                                                     \
    OR_PAR2                                                                  \
    for (int k = 0; k < (g)->n[2]; ++k)                                      \
        for (int j = 0; j < (g)->n[1]; ++j)                                  \
            for (int i = 0; i < (g)->n[0]; ++i)

/* The same walk on one thread, for the order-dependent FP64 sums. */
#define OR_LOOP_PHYS_SEQ(g)                                                  \
    int sx = (g)->n[0] + 2 * (g)->ghost, sy = (g)->n[1] + 2 * (g)->ghost;    \
    int gh = (g)->ghost;                                                     \
    for (int k = 0; k < (g)->n[2]; ++k)                                      \
        for (int j = 0; j < (g)->n[1]; ++j)                                  \
            for (int i = 0; i < (g)->n[0]; ++i)

#define OR_IDX(i, j, k) ((long)((i) + gh) + (long)sx * ((long)((j) + gh) + (long)sy * ((k) + gh)))

static inline REAL FN(lap_at)(const REAL* s, long c, long ox, long oy, long oz,
                              int dim, REAL i2x, REAL i2y, REAL i2z, int mode) {
    /* val = (f[+x] - 2f + f[-x])*i2x [+ (f[+y] - 2f + f[-y])*i2y] [+ ...z]
     * (Equation.cu:65-76).  2*f is exact, so f[+] - 2f rounds once in every
     * build.  Mode 1 contracts the y (z) product into the running sum; mode 2
     * contracts the x product with the rounded y product, the other legal
     * contraction of the same source expression. */
    REAL sc2 = (REAL)2 * s[c];
    REAL t = (s[c + ox] - sc2) + s[c - ox];
    if (dim >= 2 && mode == 2) {
        REAL t2 = (s[c + oy] - sc2) + s[c - oy];
        volatile REAL p2 = t2 * i2y;
        REAL v = FMA(t, i2x, p2);
        if (dim >= 3) { REAL t3 = (s[c + oz] - sc2) + s[c - oz]; v = FMA(t3, i2z, v); }
        return v;
    }
    volatile REAL px = t * i2x;
    REAL v = px;
    if (dim >= 2) { t = (s[c + oy] - sc2) + s[c - oy]; v = FN(madd)(mode, t, i2y, v); }
    if (dim >= 3) { t = (s[c + oz] - sc2) + s[c - oz]; v = FN(madd)(mode, t, i2z, v); }
    return v;
}

static void FN(inv_d2)(const or_grid_t* g, REAL* i2) {
    /* lap() captures 1/(d*d) in double (Equation.cu:141-143). */
    for (int a = 0; a < 3; ++a)
        i2[a] = (a < g->dim) ? (REAL)(1.0 / (g->d[a] * g->d[a])) : (REAL)0;
}

void FN(or_lap_acc)(REAL* rhs, const REAL* src, double coeff, const or_grid_t* g) {
    REAL i2[3]; FN(inv_d2)(g, i2);
    int mode = g->fma_mode;
    OR_LOOP_PHYS(g) {
        long c = OR_IDX(i, j, k);
        REAL v = FN(lap_at)(src, c, 1, sx, (long)sx * sy, g->dim, i2[0], i2[1], i2[2], mode);
        rhs[c] = FN(madd)(mode, (REAL)coeff, v, rhs[c]);
    }
}

void FN(or_grad_acc)(REAL* rhs, const REAL* src, double coeff, int axis, const or_grid_t* g) {
    REAL inv2d = (REAL)(0.5 / g->d[axis]);
    int mode = g->fma_mode;
    OR_LOOP_PHYS(g) {
        long c = OR_IDX(i, j, k);
        long o = axis == 0 ? 1 : axis == 1 ? sx : (long)sx * sy;
        /* rhs += coeff * (f[+] - f[-]) * inv_2d  ==  rhs + (coeff*diff)*inv_2d */
        REAL p = (REAL)coeff * (src[c + o] - src[c - o]);
        rhs[c] = FN(madd)(mode, p, inv2d, rhs[c]);
    }
}

/* dst[i] = fma(coeff, src[i], dst[i]) over n elements (kernel_axpy,
 * Solver.cu:30-35, as the contracted device build computes it). */
void FN(or_axpy)(REAL* dst, const REAL* src, double coeff, long n, int mode) {
    OR_PAR
    for (long i = 0; i < n; ++i) dst[i] = FN(madd)(mode, (REAL)coeff, src[i], dst[i]);
}

/* ---------------------------------------------------------------------------
 * Pointwise functors (the user lambdas of the reference's drivers).
 * ------------------------------------------------------------------------- */
static inline REAL FN(f_ac)(REAL p, int mode) {
    /* tutorials/quickstart/main.cu:66   p - p*p*p */
    REAL pp = p * p;
    return FN(madd)(mode, -pp, p, p);
}
static inline REAL FN(f_dw)(REAL c, const double* prm, int mode) {
    /* Cahn-Hillard_double-well.cu:86-92   2 rho (c-ca)(c-cb)(2c-ca-cb) */
    (void)mode;
    REAL rho = (REAL)prm[2], ca = (REAL)prm[3], cb = (REAL)prm[4];
    REAL two_rho = (REAL)2 * rho;
    return ((two_rho * (c - ca)) * (c - cb)) * (((REAL)2 * c - ca) - cb);
}
/* Coupled CH+AC bulk derivatives with f = c^2(1-c)^2 + eta^2(1-eta)^2 + lam c^2 eta^2.
 * Written with an explicit fma so host and device agree in every build. */
static inline REAL FN(f_chac_c)(REAL c, REAL e, REAL lam) {
    REAL a = (((REAL)2 * c) * ((REAL)1 - c)) * ((REAL)1 - (REAL)2 * c);
    REAL b = (((REAL)2 * lam) * c) * e;
    return FMA(b, e, a);
}
static inline REAL FN(f_chac_e)(REAL e, REAL c, REAL lam) {
    REAL a = (((REAL)2 * e) * ((REAL)1 - e)) * ((REAL)1 - (REAL)2 * e);
    REAL b = (((REAL)2 * lam) * c) * c;
    return FMA(b, e, a);
}

void FN(or_pw_acc)(REAL* rhs, const REAL* s1, const REAL* s2, double coeff,
                   int func, const double* prm, const or_grid_t* g) {
    int mode = g->fma_mode;
    OR_LOOP_PHYS(g) {
        long c = OR_IDX(i, j, k);
        REAL v;
        switch (func) {
            case OR_PW_IDENT: v = s1[c]; break;
            case OR_PW_AC:    v = FN(f_ac)(s1[c], mode); break;
            case OR_PW_DW:    v = FN(f_dw)(s1[c], prm, mode); break;
            case OR_PW_CHAC_C: v = FN(f_chac_c)(s1[c], s2[c], (REAL)prm[4]); break;
            case OR_PW_CHAC_E: v = FN(f_chac_e)(s1[c], s2[c], (REAL)prm[4]); break;
            case OR_PW_MUL:   v = s1[c] * s2[c]; break;
            default: v = 0; break;
        }
        /* TermPW.inl:36   rhs[idx] += coeff * func(src[idx]) */
        rhs[c] = FN(madd)(mode, (REAL)coeff, v, rhs[c]);
    }
}

/* Equation.cu:386-404   rhs[idx] += coeff * s1[idx] * s2[idx] */
void FN(or_mul_acc)(REAL* rhs, const REAL* s1, const REAL* s2, double coeff, const or_grid_t* g) {
    int mode = g->fma_mode;
    OR_LOOP_PHYS(g) {
        long c = OR_IDX(i, j, k);
        rhs[c] = FN(madd)(mode, (REAL)coeff * s1[c], s2[c], rhs[c]);
    }
}

/* ---------------------------------------------------------------------------
 * Equation right-hand sides, one per physics.  Each is Equation::computeRHS
 * (Equation.cu:257-276): zero the whole stored rhs, then every term's
 * accumulate in DSL order.  Composite lap(expr, bcs) is makeStencilOnExprTerm
 * (Equation.cu:537-594): zeroed scratch, materialise expr, BCs on the scratch,
 * then the stencil.
 *   prm layout per physics:
 *     AC   : [L, kappa]
 *     CH   : [M, kappa, rho, ca, cb]
 *     CHAC : [M, L, kappa_c, kappa_eta, lambda]
 * ------------------------------------------------------------------------- */
static void FN(zero)(REAL* a, long n) {
    OR_PAR
    for (long i = 0; i < n; ++i) a[i] = 0;
}

static long FN(stored)(const or_grid_t* g) {
    return (long)(g->n[0] + 2 * g->ghost) * (g->n[1] + 2 * g->ghost) * (g->n[2] + 2 * g->ghost);
}

void FN(or_rhs)(REAL** rhs, REAL** u, int phys, const double* prm,
                const or_grid_t* g, REAL* scratch) {
    long S = FN(stored)(g);
    if (phys == OR_PHYS_AC) {
        /* L*kappa*lap(phi) + L*pw(phi, p - p^3) */
        FN(zero)(rhs[0], S);
        FN(or_lap_acc)(rhs[0], u[0], prm[0] * prm[1], g);
        FN(or_pw_acc)(rhs[0], u[0], 0, prm[0], OR_PW_AC, prm, g);
    } else if (phys == OR_PHYS_CH) {
        /* M*lap(pw(c, f') - kappa*lap(c), bcs) */
        FN(zero)(rhs[0], S);
        FN(zero)(scratch, S);
        FN(or_pw_acc)(scratch, u[0], 0, 1.0, OR_PW_DW, prm, g);
        FN(or_lap_acc)(scratch, u[0], -prm[1], g);
        FN(or_bc_apply)(scratch, g);
        FN(or_lap_acc)(rhs[0], scratch, prm[0], g);
    } else if (phys == OR_PHYS_CHAC) {
        /* c  : M*lap(pw(c, eta, f_c) - kappa_c*lap(c), bcs)
         * eta: (-L)*pw(eta, c, f_eta) + (L*kappa_eta)*lap(eta) */
        FN(zero)(rhs[0], S);
        FN(zero)(scratch, S);
        FN(or_pw_acc)(scratch, u[0], u[1], 1.0, OR_PW_CHAC_C, prm, g);
        FN(or_lap_acc)(scratch, u[0], -prm[2], g);
        FN(or_bc_apply)(scratch, g);
        FN(or_lap_acc)(rhs[0], scratch, prm[0], g);
        FN(zero)(rhs[1], S);
        FN(or_pw_acc)(rhs[1], u[1], u[0], -prm[1], OR_PW_CHAC_E, prm, g);
        FN(or_lap_acc)(rhs[1], u[1], prm[1] * prm[3], g);
    }
}

static int FN(nfields)(int phys) { return phys == OR_PHYS_CHAC ? 2 : 1; }

/* ---------------------------------------------------------------------------
 * Time integration with the reference GPU solver's semantics.
 *   Euler : Solver::advance (Solver.cu:366-382) -> BCs, computeRHS,
 *           kernel_axpy over the stored array (Solver.cu:30-35, :162-168).
 *   RK4   : Solver::rk4AdvanceGPU (Solver.cu:209-259) / VectorSolver
 *           (VectorSolver.cu:149-228): stage state = phi + a*k over the whole
 *           stored array (kernel_rk4_tmp), BCs applied to the stage state,
 *           all components swapped together, then kernel_rk4_update.
 * u[f] are stored arrays (modified in place), nsteps >= 0.
 * ------------------------------------------------------------------------- */
int FN(or_advance)(REAL** u, int phys, const double* prm, int scheme,
                   double dt, int nsteps, const or_grid_t* g) {
    long S = FN(stored)(g);
    int nf = FN(nfields)(phys), mode = g->fma_mode;
    REAL* buf = (REAL*)calloc((size_t)S * (2 + 5 * nf), sizeof(REAL));
    if (!buf) return -1;
    REAL* scratch = buf;
    REAL *k1[2], *k2[2], *k3[2], *k4[2], *tmp[2];
    for (int f = 0; f < nf; ++f) {
        k1[f] = buf + S * (1 + 5 * f + 0);
        k2[f] = buf + S * (1 + 5 * f + 1);
        k3[f] = buf + S * (1 + 5 * f + 2);
        k4[f] = buf + S * (1 + 5 * f + 3);
        tmp[f] = buf + S * (1 + 5 * f + 4);
    }
    REAL dtr = (REAL)dt;
    REAL dt2 = (REAL)(dt * 0.5), dt6 = (REAL)(dt / 6.0);
    for (int s = 0; s < nsteps; ++s) {
        for (int f = 0; f < nf; ++f) FN(or_bc_apply)(u[f], g);
        if (scheme == OR_EULER) {
            FN(or_rhs)(k1, u, phys, prm, g, scratch);
            for (int f = 0; f < nf; ++f) {
                OR_PAR
                for (long i = 0; i < S; ++i) u[f][i] = FN(madd)(mode, dtr, k1[f][i], u[f][i]);
            }
            continue;
        }
        FN(or_rhs)(k1, u, phys, prm, g, scratch);
        REAL** ks[3] = {k1, k2, k3};
        REAL** kn[3] = {k2, k3, k4};
        REAL as[3] = {dt2, dt2, dtr};
        for (int st = 0; st < 3; ++st) {
            for (int f = 0; f < nf; ++f) {
                OR_PAR
                for (long i = 0; i < S; ++i) tmp[f][i] = FN(madd)(mode, as[st], ks[st][f][i], u[f][i]);
                FN(or_bc_apply)(tmp[f], g);
            }
            FN(or_rhs)(kn[st], tmp, phys, prm, g, scratch);
        }
        for (int f = 0; f < nf; ++f) {
            OR_PAR
            for (long i = 0; i < S; ++i) {
                REAL a = (k1[f][i] + (REAL)2 * k2[f][i]) + (REAL)2 * k3[f][i];
                a = a + k4[f][i];
                u[f][i] = FN(madd)(mode, dt6, a, u[f][i]);
            }
        }
    }
    free(buf);
    return 0;
}

/* ---------------------------------------------------------------------------
 * Compensated state (the FP32 kernels' scheme): the state is the unevaluated
 * sum hi + lo of two REALs.  Stage states and right-hand sides use hi only,
 * exactly as or_advance does; the final update adds delta = dt*k (Euler) or
 * dt/6*(k1+2k2+2k3+k4) (RK4) to (hi, lo) with an error-free two-sum and a
 * renormalisation, so the state itself is not rounded to REAL each step.
 * BCs refresh the ghosts of hi at the start of each step; lo never enters a
 * stencil, so its ghosts are left as they are.
 * ------------------------------------------------------------------------- */
static inline void FN(twosum_update)(REAL* h, REAL* l, REAL d) {
    volatile REAL s = *h + d;
    volatile REAL bp = s - *h;
    volatile REAL e = (*h - (s - bp)) + (d - bp);
    volatile REAL l2 = *l + e;
    volatile REAL h2 = s + l2;
    *l = l2 - (h2 - s);
    *h = h2;
}

int FN(or_advance_comp)(REAL** hi, REAL** lo, int phys, const double* prm, int scheme, double dt, int nsteps,
                        const or_grid_t* g) {
    long S = FN(stored)(g);
    int nf = FN(nfields)(phys), mode = g->fma_mode;
    REAL* buf = (REAL*)calloc((size_t)S * (2 + 5 * nf), sizeof(REAL));
    if (!buf) return -1;
    REAL* scratch = buf;
    REAL *k1[2], *k2[2], *k3[2], *k4[2], *tmp[2];
    for (int f = 0; f < nf; ++f) {
        k1[f] = buf + S * (1 + 5 * f + 0);
        k2[f] = buf + S * (1 + 5 * f + 1);
        k3[f] = buf + S * (1 + 5 * f + 2);
        k4[f] = buf + S * (1 + 5 * f + 3);
        tmp[f] = buf + S * (1 + 5 * f + 4);
    }
    REAL dtr = (REAL)dt;
    REAL dt2 = (REAL)(dt * 0.5), dt6 = (REAL)(dt / 6.0);
    for (int s = 0; s < nsteps; ++s) {
        for (int f = 0; f < nf; ++f) FN(or_bc_apply)(hi[f], g);
        FN(or_rhs)(k1, hi, phys, prm, g, scratch);
        if (scheme == OR_EULER) {
            for (int f = 0; f < nf; ++f)
                for (long i = 0; i < S; ++i) {
                    volatile REAL d = dtr * k1[f][i];
                    FN(twosum_update)(&hi[f][i], &lo[f][i], d);
                }
            continue;
        }
        REAL** ks[3] = {k1, k2, k3};
        REAL** kn[3] = {k2, k3, k4};
        REAL as[3] = {dt2, dt2, dtr};
        for (int st = 0; st < 3; ++st) {
            for (int f = 0; f < nf; ++f) {
                for (long i = 0; i < S; ++i) tmp[f][i] = FN(madd)(mode, as[st], ks[st][f][i], hi[f][i]);
                FN(or_bc_apply)(tmp[f], g);
            }
            FN(or_rhs)(kn[st], tmp, phys, prm, g, scratch);
        }
        for (int f = 0; f < nf; ++f)
            for (long i = 0; i < S; ++i) {
                REAL a = (k1[f][i] + (REAL)2 * k2[f][i]) + (REAL)2 * k3[f][i];
                a = a + k4[f][i];
                volatile REAL d = dt6 * a;
                FN(twosum_update)(&hi[f][i], &lo[f][i], d);
            }
    }
    free(buf);
    return 0;
}

/* ---------------------------------------------------------------------------
 * Multi-step Euler (Solver.cu:317-340) for the shipped Cahn-Hilliard app
 * (Cahn-Hillard_double-well.cu:84-106):
 *   step 1 (STEADY)   : BCs on c, mu = pw(c, f') - kappa*lap(c)
 *   step 2 (TRANSIENT): BCs on mu, c += dt * (M*lap(mu))
 * prm = [M, kappa, rho, ca, cb]; c and mu are stored arrays.
 * ------------------------------------------------------------------------- */
int FN(or_advance_ch_multistep)(REAL* c, REAL* mu, const double* prm, double dt,
                                int nsteps, const or_grid_t* g) {
    long S = FN(stored)(g);
    int mode = g->fma_mode;
    REAL* rhs = (REAL*)calloc((size_t)S, sizeof(REAL));
    if (!rhs) return -1;
    for (int s = 0; s < nsteps; ++s) {
        FN(or_bc_apply)(c, g);
        FN(zero)(mu, S);
        FN(or_pw_acc)(mu, c, 0, 1.0, OR_PW_DW, prm, g);
        FN(or_lap_acc)(mu, c, -prm[1], g);
        FN(or_bc_apply)(mu, g);
        FN(zero)(rhs, S);
        FN(or_lap_acc)(rhs, mu, prm[0], g);
        OR_PAR
        for (long i = 0; i < S; ++i) c[i] = FN(madd)(mode, (REAL)dt, rhs[i], c[i]);
    }
    free(rhs);
    return 0;
}

/* ---------------------------------------------------------------------------
 * Diagnostics, accumulated in double in x-fastest order.
 *   mass   = sum_phys c * dV
 *   energy = sum_phys [ f(c) + kappa/2 |grad c|^2 ] * dV, central gradient on
 *            BC-filled ghosts (develop/Spinodal Decomposition/
 *            computeFreeEnergy.py:76-98; np.roll == periodic ghosts).
 * The field's ghosts are filled on a private copy; the input is not touched.
 * ------------------------------------------------------------------------- */
static double FN(dvol)(const or_grid_t* g) {
    double v = 1.0;
    for (int a = 0; a < g->dim; ++a) v *= g->d[a];
    return v;
}

double FN(or_mass)(const REAL* u, const or_grid_t* g) {
    double s = 0.0;
    OR_LOOP_PHYS_SEQ(g) { s += (double)u[OR_IDX(i, j, k)]; }
    return s * FN(dvol)(g);
}

double FN(or_energy)(REAL** u_in, int phys, const double* prm, const or_grid_t* g) {
    long S = FN(stored)(g);
    int nf = FN(nfields)(phys);
    REAL* w = (REAL*)malloc(sizeof(REAL) * S * nf);
    if (!w) return NAN;
    REAL* u[2];
    for (int f = 0; f < nf; ++f) {
        u[f] = w + S * f;
        memcpy(u[f], u_in[f], sizeof(REAL) * S);
        FN(or_bc_apply)(u[f], g);
    }
    double kap[2];
    if (phys == OR_PHYS_AC) kap[0] = prm[1];
    else if (phys == OR_PHYS_CH) kap[0] = prm[1];
    else { kap[0] = prm[2]; kap[1] = prm[3]; }
    double tot = 0.0;
    OR_LOOP_PHYS_SEQ(g) {
        long c = OR_IDX(i, j, k);
        long off[3] = {1, sx, (long)sx * sy};
        double fb;
        if (phys == OR_PHYS_AC) {
            double p = u[0][c];
            fb = 0.25 * (p * p - 1.0) * (p * p - 1.0);
        } else if (phys == OR_PHYS_CH) {
            double x = u[0][c], rho = prm[2], ca = prm[3], cb = prm[4];
            fb = rho * (x - ca) * (x - ca) * (cb - x) * (cb - x);
        } else {
            double x = u[0][c], e = u[1][c], lam = prm[4];
            fb = x * x * (1.0 - x) * (1.0 - x) + e * e * (1.0 - e) * (1.0 - e) + lam * x * x * e * e;
        }
        double gr = 0.0;
        for (int f = 0; f < nf; ++f) {
            double g2 = 0.0;
            for (int a = 0; a < g->dim; ++a) {
                double d = ((double)u[f][c + off[a]] - (double)u[f][c - off[a]]) / (2.0 * g->d[a]);
                g2 += d * d;
            }
            gr += 0.5 * kap[f] * g2;
        }
        tot += fb + gr;
    }
    free(w);
    return tot * FN(dvol)(g);
}

#undef OR_LOOP_PHYS
#undef OR_LOOP_PHYS_SEQ
#undef OR_IDX
#undef FN
#undef CAT
#undef CAT_
