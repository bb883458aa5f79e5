// stepper.cu -- fused time stepper behind phix_stepper_* (Solver / VectorSolver
// replacement, Solver.cu:86-259, VectorSolver.cu:77-228).
//
// RK4 step = 4 launches:
//   stage 1: k1 = F(u)                       (BCs folded into halo loads)
//   stage 2: k2 = F(u + dt/2 k1)
//   stage 3: k3 = F(u + dt/2 k2)
//   stage 4: u' = u + dt/6 (k1 + 2k2 + 2k3 + F(u + dt k3))   -> other state buffer
// Euler step = 1 launch: u' = u + dt F(u).
// The state ping-pongs between two buffers; k buffers are per field.  Groups
// of steps can be captured once into a CUDA graph and replayed.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <algorithm>
#include <utility>
#include <vector>

#include "phix/detail/common.cuh"
#include "phix/detail/stage.cuh"
#include "phix/detail/stage_col.cuh"
#include "phix/detail/step2d.cuh"
#include "phix/detail/step2d_pair.cuh"
#include "phix/detail/step2d_pair_ms.cuh"
#include "phix/detail/march3d_fused.cuh"
#include "phix/detail/stream3d.cuh"
#include "stepper.h"

#include <cudaTypedefs.h>

namespace phix {

// ---------------------------------------------------------------------------
// launch dispatch
// ---------------------------------------------------------------------------
namespace {

constexpr int BOX_TX = 64, BOX_TY = 16, BOX_NT = 256;
constexpr int LIN_TX = 256, LIN_NT = 256;
constexpr int M3_TX = 32, M3_TY = 8, M3_RZ = 16, M3_NT = 256;

// 2-D column-walking tiles (stage_col.cuh): (TX, TY, row groups G); TX*G threads.
constexpr int kColCfgs[][3] = {{64, 16, 4}, {64, 32, 4}, {128, 16, 2}, {32, 16, 8}};
constexpr int kNumColCfgs = sizeof(kColCfgs) / sizeof(kColCfgs[0]);

template <typename T, class Pol, int MODE, int TX, int TY, int G>
int launch_col_cfg(const StageArgs<T>& A, cudaStream_t s) {
    dim3 grid((A.L.n[0] + TX - 1) / TX, (A.L.n[1] + TY - 1) / TY, 1);
    stage_col<T, Pol, MODE, TX, TY, G><<<grid, TX * G, col_smem_bytes<T, Pol, TX, TY>(), s>>>(A, Pol{});
    PHIX_LAUNCH_CHECK("stage_col");
    return PHIX_OK;
}

template <typename T, class Pol, int MODE, int TX, int TY, int G>
int prepare_col_cfg() {
    PHIX_TRY_CUDA(cudaFuncSetAttribute(stage_col<T, Pol, MODE, TX, TY, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)col_smem_bytes<T, Pol, TX, TY>()));
    return PHIX_OK;
}

template <typename T, class Pol, int MODE>
int col_dispatch(int cfg, bool prepare, const StageArgs<T>* A, cudaStream_t s) {
    switch (cfg) {
#define PHIX_COL_CASE(i)                                                                         \
    case i:                                                                                      \
        return prepare ? prepare_col_cfg<T, Pol, MODE, kColCfgs[i][0], kColCfgs[i][1], kColCfgs[i][2]>()  \
                       : launch_col_cfg<T, Pol, MODE, kColCfgs[i][0], kColCfgs[i][1], kColCfgs[i][2]>(*A, s);
        PHIX_COL_CASE(0)
        PHIX_COL_CASE(1)
        PHIX_COL_CASE(2)
        PHIX_COL_CASE(3)
#undef PHIX_COL_CASE
    }
    set_error("stage: bad 2-D tile configuration %d", cfg);
    return PHIX_ERR_ARG;
}

template <typename T, int PHYS, int DIM, int MODE>
int launch_box(const StageArgs<T>& A, cudaStream_t s, int tile) {
    using Pol = typename PolOf<PHYS>::type;
    if constexpr (DIM == 2 && MODE != MODE_MULTISTEP) {
        if (tile >= 0) return col_dispatch<T, Pol, MODE>(tile, false, &A, s);
    }
    if (DIM == 1) {
        dim3 grid((A.L.n[0] + LIN_TX - 1) / LIN_TX, 1, 1);
        stage_box<T, Pol, 1, MODE, LIN_TX, 1, LIN_NT><<<grid, LIN_NT, 0, s>>>(A, Pol{});
    } else {
        dim3 grid((A.L.n[0] + BOX_TX - 1) / BOX_TX, (A.L.n[1] + BOX_TY - 1) / BOX_TY, 1);
        stage_box<T, Pol, 2, MODE, BOX_TX, BOX_TY, BOX_NT><<<grid, BOX_NT, 0, s>>>(A, Pol{});
    }
    PHIX_LAUNCH_CHECK("stage_box");
    return PHIX_OK;
}

// Dynamic shared memory of the 3-D kernels is opted in once per stepper
// creation (never inside a stream capture).
template <typename T, int PHYS, int MODE>
int prepare_march() {
    using Pol = typename PolOf<PHYS>::type;
    using G = March3D<T, Pol, M3_TX, M3_TY>;
    auto kern = stage_march3d<T, Pol, MODE, M3_TX, M3_TY, M3_RZ, M3_NT>;
    PHIX_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::smem_bytes()));
    return PHIX_OK;
}

template <typename T, int PHYS>
int prepare_phys() {
    int rc;
    if ((rc = prepare_march<T, PHYS, MODE_K>())) return rc;
    if ((rc = prepare_march<T, PHYS, MODE_RK4_FINAL>())) return rc;
    return prepare_march<T, PHYS, MODE_EULER_FINAL>();
}

template <typename T>
int prepare_t(int phys) {
    switch (phys) {
        case PHIX_PHYS_AC: return prepare_phys<T, PHIX_PHYS_AC>();
        case PHIX_PHYS_CH: return prepare_phys<T, PHIX_PHYS_CH>();
        default: return prepare_phys<T, PHIX_PHYS_CHAC>();
    }
}

template <typename T, int PHYS, int MODE>
int launch_march(const StageArgs<T>& A, cudaStream_t s) {
    using Pol = typename PolOf<PHYS>::type;
    using G = March3D<T, Pol, M3_TX, M3_TY>;
    auto kern = stage_march3d<T, Pol, MODE, M3_TX, M3_TY, M3_RZ, M3_NT>;
    const size_t smem = G::smem_bytes();
    dim3 grid((A.L.n[0] + M3_TX - 1) / M3_TX, (A.L.n[1] + M3_TY - 1) / M3_TY, (A.L.n[2] + M3_RZ - 1) / M3_RZ);
    kern<<<grid, M3_NT, smem, s>>>(A, Pol{});
    PHIX_LAUNCH_CHECK("stage_march3d");
    return PHIX_OK;
}

template <typename T, int PHYS, int MODE>
int launch_dim(int dim, const StageArgs<T>& A, cudaStream_t s, int tile) {
    switch (dim) {
        case 1: return launch_box<T, PHYS, 1, MODE>(A, s, tile);
        case 2: return launch_box<T, PHYS, 2, MODE>(A, s, tile);
        case 3: return launch_march<T, PHYS, MODE>(A, s);
    }
    set_error("stage: unsupported dim %d", dim);
    return PHIX_ERR_ARG;
}

template <typename T, int PHYS>
int launch_mode(int dim, int mode, const StageArgs<T>& A, cudaStream_t s, int tile) {
    switch (mode) {
        case MODE_K: return launch_dim<T, PHYS, MODE_K>(dim, A, s, tile);
        case MODE_RK4_FINAL: return launch_dim<T, PHYS, MODE_RK4_FINAL>(dim, A, s, tile);
        case MODE_EULER_FINAL: return launch_dim<T, PHYS, MODE_EULER_FINAL>(dim, A, s, tile);
        case MODE_MULTISTEP:
            if (PHYS == PHIX_PHYS_CH && dim <= 2) {
                if (dim == 1) return launch_box<T, PHIX_PHYS_CH, 1, MODE_MULTISTEP>(A, s, -1);
                return launch_box<T, PHIX_PHYS_CH, 2, MODE_MULTISTEP>(A, s, -1);
            }
            break;
    }
    set_error("stage: bad mode %d", mode);
    return PHIX_ERR_ARG;
}

// ---------------------------------------------------------------------------
// one launch per RK4 step (2-D, one field)
// ---------------------------------------------------------------------------
// tiles of the one-launch step: (TX, TY, threads); index 0 is the default
constexpr int kStepCfgs[][3] = {{64, 16, 256}, {64, 32, 256}, {128, 16, 256}, {128, 32, 512}, {128, 64, 1024},
                                 {256, 32, 1024}};
constexpr size_t kMaxSmem = 227 * 1024;  // opt-in shared memory per CTA on sm_100
constexpr int kNumStepCfgs = sizeof(kStepCfgs) / sizeof(kStepCfgs[0]);
// tiles of the pair kernels (CH, four periodic sides): (TX, TY, row blocks,
// time steps per launch); threads = (TX / 2 + 8 depth) x row blocks.  Step
// configuration kNumStepCfgs + i.  The last four are temporally blocked:
// two RK4 steps per launch on a tile with a 16-cell halo.
constexpr int kPairCfgs[][4] = {{128, 64, 8, 1}, {128, 32, 8, 1}, {128, 32, 4, 1}, {128, 16, 4, 1}, {64, 32, 8, 1},
                                 {64, 64, 8, 1},  {256, 32, 4, 1}, {128, 28, 8, 1}, {64, 28, 8, 1},  {64, 16, 4, 1},
                                 {64, 32, 8, 2},  {64, 16, 4, 2},  {128, 16, 4, 2}, {64, 28, 8, 2}};
constexpr int kNumPairCfgs = sizeof(kPairCfgs) / sizeof(kPairCfgs[0]);

template <typename T, class Pol, int TX, int TY, int NT>
int step_cfg(bool prepare, const StepArgs<T>* A, cudaStream_t s) {
    using G = Step2D<T, Pol, TX, TY>;
    if (G::smem_bytes() > kMaxSmem) {  // this tile does not fit for this type / physics
        if (prepare) return PHIX_OK;
        set_error("step2d: a %dx%d tile needs %zu bytes of shared memory", TX, TY, G::smem_bytes());
        return PHIX_ERR_UNSUPPORTED;
    }
    if (prepare) {
        PHIX_TRY_CUDA(cudaFuncSetAttribute(step_box<T, Pol, TX, TY, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)G::smem_bytes()));
        return PHIX_OK;
    }
    dim3 grid((A->S.L.n[0] + TX - 1) / TX, (A->S.L.n[1] + TY - 1) / TY, 1);
    step_box<T, Pol, TX, TY, NT><<<grid, NT, G::smem_bytes(), s>>>(*A, Pol{});
    PHIX_LAUNCH_CHECK("step_box");
    return PHIX_OK;
}

template <typename T, int PHYS>
int step_dispatch(int cfg, bool prepare, const StepArgs<T>* A, cudaStream_t s) {
    using Pol = typename PolOf<PHYS>::type;
    switch (cfg) {
#define PHIX_STEP_CASE(i) \
    case i: return step_cfg<T, Pol, kStepCfgs[i][0], kStepCfgs[i][1], kStepCfgs[i][2]>(prepare, A, s);
        PHIX_STEP_CASE(0)
        PHIX_STEP_CASE(1)
        PHIX_STEP_CASE(2)
        PHIX_STEP_CASE(3)
        PHIX_STEP_CASE(4)
        PHIX_STEP_CASE(5)
#undef PHIX_STEP_CASE
    }
    set_error("step2d: bad tile configuration %d", cfg);
    return PHIX_ERR_ARG;
}

// prepare: set the shared-memory attribute; occ != nullptr: report resident
// CTAs per SM (0: does not fit); else launch.
template <typename T, int TX, int TY, int NRP, int NS>
int pair_cfg(bool prepare, const StepArgs<T>* A, cudaStream_t s, int* occ = nullptr) {
    using G = StepPair<T, TX, TY, NRP, NS>;
    if (G::smem_bytes() > kMaxSmem) {
        if (occ) *occ = 0;
        if (prepare || occ) return PHIX_OK;
        set_error("step_pair: a %dx%d tile needs %zu bytes of shared memory", TX, TY, G::smem_bytes());
        return PHIX_ERR_UNSUPPORTED;
    }
    if (occ) {
        PHIX_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, step_pair<T, PolCH, TX, TY, NRP, NS>, G::NT,
                                                                    G::smem_bytes()));
        return PHIX_OK;
    }
    if (prepare) {
        PHIX_TRY_CUDA(cudaFuncSetAttribute(step_pair<T, PolCH, TX, TY, NRP, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)G::smem_bytes()));
        return PHIX_OK;
    }
    dim3 grid((A->S.L.n[0] + TX - 1) / TX, (A->S.L.n[1] + TY - 1) / TY, 1);
    // launched one by one (not into a graph), each step is a programmatic
    // dependent of the previous launch on the stream: its CTAs are scheduled
    // while the previous step's last wave runs and wait in the kernel
    // (griddepcontrol.wait) for that step's writes.  Graph replays keep plain
    // edges: dependent launches measured 1-3 % slower there.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    PHIX_TRY_CUDA(cudaStreamIsCapturing(s, &cap));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(G::NT);
    cfg.dynamicSmemBytes = G::smem_bytes();
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = cap == cudaStreamCaptureStatusNone ? 1 : 0;
    cudaError_t e = cudaLaunchKernelEx(&cfg, step_pair<T, PolCH, TX, TY, NRP, NS>, *A, PolCH{});
    if (e == cudaErrorNotSupported || e == cudaErrorInvalidValue) {
        (void)cudaGetLastError();  // a stream without dependent launches: an ordinary launch
        cfg.numAttrs = 0;
        e = cudaLaunchKernelEx(&cfg, step_pair<T, PolCH, TX, TY, NRP, NS>, *A, PolCH{});
    }
    if (e != cudaSuccess) return cuda_status(e, "step_pair launch");
    PHIX_LAUNCH_CHECK("step_pair");
    return PHIX_OK;
}

template <typename T>
int pair_dispatch(int i, bool prepare, const StepArgs<T>* A, cudaStream_t s, int* occ = nullptr) {
    switch (i) {
#define PHIX_PAIR_CASE(i) \
    case i: return pair_cfg<T, kPairCfgs[i][0], kPairCfgs[i][1], kPairCfgs[i][2], kPairCfgs[i][3]>(prepare, A, s, occ);
        PHIX_PAIR_CASE(0)
        PHIX_PAIR_CASE(1)
        PHIX_PAIR_CASE(2)
        PHIX_PAIR_CASE(3)
        PHIX_PAIR_CASE(4)
        PHIX_PAIR_CASE(5)
        PHIX_PAIR_CASE(6)
        PHIX_PAIR_CASE(7)
        PHIX_PAIR_CASE(8)
        PHIX_PAIR_CASE(9)
        PHIX_PAIR_CASE(10)
        PHIX_PAIR_CASE(11)
        PHIX_PAIR_CASE(12)
        PHIX_PAIR_CASE(13)
#undef PHIX_PAIR_CASE
    }
    set_error("step_pair: bad tile configuration %d", i);
    return PHIX_ERR_ARG;
}

// tiles of the multi-step pair kernel (CH, four periodic sides): (TX, TY,
// row blocks); threads = (TX / 2 + 2) x row blocks.
constexpr int kMsCfgs[][3] = {{128, 32, 8}, {64, 32, 8}, {128, 16, 4}, {64, 16, 4}, {64, 64, 8}, {256, 16, 4}};
constexpr int kNumMsCfgs = sizeof(kMsCfgs) / sizeof(kMsCfgs[0]);

// prepare: set the shared-memory attribute; occ != nullptr: report resident
// CTAs per SM; else launch.
template <typename T, int TX, int TY, int NRP>
int ms_cfg(bool prepare, const StageArgs<T>* A, cudaStream_t s, int* occ = nullptr) {
    using G = MsPair<T, TX, TY, NRP>;
    static_assert(G::smem_bytes() <= kMaxSmem, "multi-step pair tile too large");
    auto kern = step_pair_ms<T, PolCH, TX, TY, NRP>;
    if (occ) {
        PHIX_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, kern, G::NT, G::smem_bytes()));
        return PHIX_OK;
    }
    if (prepare) {
        PHIX_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::smem_bytes()));
        return PHIX_OK;
    }
    dim3 grid((A->L.n[0] + TX - 1) / TX, (A->L.n[1] + TY - 1) / TY, 1);
    kern<<<grid, G::NT, G::smem_bytes(), s>>>(*A, PolCH{});
    PHIX_LAUNCH_CHECK("step_pair_ms");
    return PHIX_OK;
}

template <typename T>
int ms_dispatch(int i, bool prepare, const StageArgs<T>* A, cudaStream_t s, int* occ = nullptr) {
    switch (i) {
#define PHIX_MS_CASE(i) \
    case i: return ms_cfg<T, kMsCfgs[i][0], kMsCfgs[i][1], kMsCfgs[i][2]>(prepare, A, s, occ);
        PHIX_MS_CASE(0)
        PHIX_MS_CASE(1)
        PHIX_MS_CASE(2)
        PHIX_MS_CASE(3)
        PHIX_MS_CASE(4)
        PHIX_MS_CASE(5)
#undef PHIX_MS_CASE
    }
    set_error("step_pair_ms: bad tile configuration %d", i);
    return PHIX_ERR_UNSUPPORTED;
}

template <typename T, int PHYS>
int prepare_step2d_t() {
    for (int c = 0; c < kNumStepCfgs; ++c) {
        int rc = step_dispatch<T, PHYS>(c, true, nullptr, 0);
        if (rc) return rc;
    }
    if (PHYS == PHIX_PHYS_CH) {
        for (int c = 0; c < kNumPairCfgs; ++c) {
            int rc = pair_dispatch<T>(c, true, nullptr, 0);
            if (rc) return rc;
        }
        for (int c = 0; c < kNumMsCfgs; ++c) {
            int rc = ms_dispatch<T>(c, true, nullptr, 0);
            if (rc) return rc;
        }
    }
    return PHIX_OK;
}

}  // namespace

template <typename T, int PHYS>
int prepare_col_t() {
    using Pol = typename PolOf<PHYS>::type;
    for (int c = 0; c < kNumColCfgs; ++c) {
        int rc;
        if ((rc = col_dispatch<T, Pol, MODE_K>(c, true, nullptr, 0))) return rc;
        if ((rc = col_dispatch<T, Pol, MODE_RK4_FINAL>(c, true, nullptr, 0))) return rc;
        if ((rc = col_dispatch<T, Pol, MODE_EULER_FINAL>(c, true, nullptr, 0))) return rc;
    }
    return PHIX_OK;
}

int prepare_stage(int phys, int dim, int prec) {
    if (dim == 2) {
        int rc;
        if (prec == PHIX_F32)
            rc = phys == PHIX_PHYS_AC ? prepare_col_t<float, PHIX_PHYS_AC>()
               : phys == PHIX_PHYS_CH ? prepare_col_t<float, PHIX_PHYS_CH>() : prepare_col_t<float, PHIX_PHYS_CHAC>();
        else
            rc = phys == PHIX_PHYS_AC ? prepare_col_t<double, PHIX_PHYS_AC>()
               : phys == PHIX_PHYS_CH ? prepare_col_t<double, PHIX_PHYS_CH>() : prepare_col_t<double, PHIX_PHYS_CHAC>();
        if (rc) return rc;
    }
    if (dim == 2 && (phys == PHIX_PHYS_AC || phys == PHIX_PHYS_CH)) {
        int rc;
        if (prec == PHIX_F32)
            rc = phys == PHIX_PHYS_AC ? prepare_step2d_t<float, PHIX_PHYS_AC>() : prepare_step2d_t<float, PHIX_PHYS_CH>();
        else
            rc = phys == PHIX_PHYS_AC ? prepare_step2d_t<double, PHIX_PHYS_AC>()
                                      : prepare_step2d_t<double, PHIX_PHYS_CH>();
        if (rc) return rc;
    }
    if (dim != 3) return PHIX_OK;
    return prec == PHIX_F32 ? prepare_t<float>(phys) : prepare_t<double>(phys);
}

// Pair tile for a grid: among the shapes with at least two resident CTAs
// and 1024 (FP32) or 512 (FP64) resident threads per SM (fewer leave too few
// warps to hide the barriers' latency), the least (tiles per SM, rounded up)
// x (work per tile), work per tile being the cells of the eight passes'
// regions; ties go to the earlier shape.  Grids that do not fill the SMs
// get smaller tiles spread over more of them.  On B200 this picks 128x28
// (FP32) and 64x28 (FP64) at 1024^2 and 128x32 for FP32 at 4096^2, the
// fastest measured there.
template <typename T>
int pick_pair_cfg(const Layout& L, int nsm) {
    int best = 1;
    double best_cost = 1e300;
    for (int i = 0; i < kNumPairCfgs; ++i) {
        if (kPairCfgs[i][3] != 1) continue;  // the default is one step per launch
        int occ = 0;
        if (pair_dispatch<T>(i, false, nullptr, 0, &occ) != PHIX_OK || occ < 2) continue;
        const int tx = kPairCfgs[i][0], ty = kPairCfgs[i][1];
        if (occ * (tx / 2 + 8) * kPairCfgs[i][2] < (sizeof(T) == 4 ? 1024 : 512)) continue;
        const double tiles = (double)((L.n[0] + tx - 1) / tx) * ((L.n[1] + ty - 1) / ty);
        double work = 0.0;
        for (int e = 0; e <= 7; ++e) work += (double)(tx + 2 * e + (e & 1)) * (ty + 2 * e);
        const double cost = std::ceil(tiles / nsm) * work;
        if (cost < best_cost) { best_cost = cost; best = i; }
    }
    return best;
}

// Default tile of the one-launch step (measured on B200): 128x32 with 512
// threads, or 128x64 with 1024 threads in FP32 when those tiles fill at most
// one wave (one CTA per SM: the smaller grids, e.g. 1024^2).
template <typename T>
int default_step_cfg(int phys, const Layout& L) {
    static int nsm = 0;
    if (!nsm) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm <= 0) nsm = 148;
    }
    if (phys == PHIX_PHYS_CH && step_pair_supported(L, 2)) return kNumStepCfgs + pick_pair_cfg<T>(L, nsm);
    if (sizeof(T) == 4) {
        const long long tiles = (long long)((L.n[0] + 127) / 128) * ((L.n[1] + 63) / 64);
        if (tiles <= nsm) return 4;
    }
    return 3;
}

// The multi-step Cahn-Hilliard step in the pair layout (CH, 2-D, four
// periodic sides); tile < 0 takes the default shape: 64x16 tiles with 4 row
// blocks, or 128x16 from 4 M cells up (the fastest measured on B200 at
// 512^2, 1024^2 and 4096^2, FP32 and FP64).
template <typename T>
int launch_ms(const StageArgs<T>& A, cudaStream_t s, int tile) {
    const int cfg = tile >= 0 ? tile : (long long)A.L.n[0] * A.L.n[1] >= (4LL << 20) ? 2 : 3;
    if (cfg >= kNumMsCfgs) {
        set_error("step_pair_ms: tile configuration %d out of range", cfg);
        return PHIX_ERR_UNSUPPORTED;
    }
    return ms_dispatch<T>(cfg, false, &A, s);
}

// Time steps one launch of step configuration `tile` advances (1, or 2 for
// the temporally blocked pair tiles).
int step_cfg_depth(int tile) {
    return tile >= kNumStepCfgs && tile < kNumStepCfgs + kNumPairCfgs ? kPairCfgs[tile - kNumStepCfgs][3] : 1;
}

// One launch advancing `depth` steps (a depth-1 launch of a depth-2
// configuration takes the grid's default single-step shape).
template <typename T>
int launch_step2d(int phys, const StepArgs<T>& A, cudaStream_t s, int tile, int depth = 1) {
    int cfg = tile < 0 ? default_step_cfg<T>(phys, A.S.L) : tile;
    if (step_cfg_depth(cfg) != depth) {
        if (depth != 1) {
            set_error("step_pair: configuration %d does not take %d steps per launch", cfg, depth);
            return PHIX_ERR_ARG;
        }
        cfg = default_step_cfg<T>(phys, A.S.L);
    }
    if (cfg >= kNumStepCfgs) {
        if (phys != PHIX_PHYS_CH || !step_pair_supported(A.S.L, 2)) {
            set_error("step_pair: tile configuration %d needs CH with four periodic sides", cfg);
            return PHIX_ERR_UNSUPPORTED;
        }
        return pair_dispatch<T>(cfg - kNumStepCfgs, false, &A, s);
    }
    if (phys == PHIX_PHYS_AC) return step_dispatch<T, PHIX_PHYS_AC>(cfg, false, &A, s);
    if (phys == PHIX_PHYS_CH) return step_dispatch<T, PHIX_PHYS_CH>(cfg, false, &A, s);
    set_error("step2d: physics %d has more than one field", phys);
    return PHIX_ERR_UNSUPPORTED;
}

template <typename T>
int launch_stage(int phys, int dim, int mode, const StageArgs<T>& A, cudaStream_t s, int tile) {
    switch (phys) {
        case PHIX_PHYS_AC: return launch_mode<T, PHIX_PHYS_AC>(dim, mode, A, s, tile);
        case PHIX_PHYS_CH: return launch_mode<T, PHIX_PHYS_CH>(dim, mode, A, s, tile);
        case PHIX_PHYS_CHAC: return launch_mode<T, PHIX_PHYS_CHAC>(dim, mode, A, s, tile);
    }
    set_error("stage: unknown physics %d", phys);
    return PHIX_ERR_ARG;
}
template int launch_stage<float>(int, int, int, const StageArgs<float>&, cudaStream_t, int);
template int launch_stage<double>(int, int, int, const StageArgs<double>&, cudaStream_t, int);

// ---------------------------------------------------------------------------
// grid validation / layout
// ---------------------------------------------------------------------------
int validate_grid(const phix_grid_t* g, Layout* L, size_t* stored) {
    if (!g) { set_error("grid is NULL"); return PHIX_ERR_ARG; }
    if (g->dim < 1 || g->dim > 3) { set_error("grid.dim must be 1, 2 or 3 (got %d)", g->dim); return PHIX_ERR_ARG; }
    if (g->ghost < 1) { set_error("grid.ghost must be >= 1 (got %d)", g->ghost); return PHIX_ERR_ARG; }
    for (int a = 0; a < 3; ++a) {
        if (g->n[a] < 1) { set_error("grid.n[%d] must be >= 1", a); return PHIX_ERR_ARG; }
        if (a >= g->dim && g->n[a] != 1) { set_error("grid.n[%d] must be 1 for unused axes", a); return PHIX_ERR_ARG; }
        if (a < g->dim && !(g->d[a] > 0.0)) { set_error("grid.d[%d] must be > 0", a); return PHIX_ERR_ARG; }
    }
    for (int i = 0; i < 6; ++i) {
        int t = g->bc_type[i];
        if (t < PHIX_BC_NONE || t > PHIX_BC_FIXED) { set_error("grid.bc_type[%d] invalid (%d)", i, t); return PHIX_ERR_ARG; }
    }
    for (int a = 0; a < g->dim; ++a) {
        bool pl = g->bc_type[2 * a] == PHIX_BC_PERIODIC, ph = g->bc_type[2 * a + 1] == PHIX_BC_PERIODIC;
        if (pl != ph) {
            set_error("Periodic BC must be set on both sides of axis %c", "XYZ"[a]);
            return PHIX_ERR_ARG;
        }
    }
    long long sx = g->n[0] + 2LL * g->ghost, sy = g->n[1] + 2LL * g->ghost, sz = g->n[2] + 2LL * g->ghost;
    long long S = sx * sy * sz;
    if (S >= (1LL << 31)) { set_error("stored size %lld exceeds 2^31 elements", S); return PHIX_ERR_ARG; }
    if (L) {
        for (int a = 0; a < 3; ++a) L->n[a] = g->n[a];
        L->s[0] = 1;
        L->s[1] = (int)sx;
        L->s[2] = (int)(sx * sy);
        L->ghost = g->ghost;
        L->origin = (int)(g->ghost + sx * (g->ghost + sy * g->ghost));
        for (int i = 0; i < 6; ++i) {
            // axes beyond dim carry no BC (their ghost planes are never read)
            L->bc[i] = (i / 2 < g->dim) ? g->bc_type[i] : PHIX_BC_NONE;
            L->bcv[i] = g->bc_val[i];
        }
    }
    if (stored) *stored = (size_t)S;
    return PHIX_OK;
}

int physics_nfields(int phys) { return phys == PHIX_PHYS_CHAC ? 2 : (phys == PHIX_PHYS_AC || phys == PHIX_PHYS_CH) ? 1 : 0; }

// Physics coefficients in kernel precision (rounded from double exactly the
// way the oracle rounds them).
template <typename T>
void make_coeffs(int phys, const double* prm, T* p) {
    for (int i = 0; i < 8; ++i) p[i] = (T)0;
    if (phys == PHIX_PHYS_AC) {
        p[0] = (T)(prm[0] * prm[1]);  // L*kappa (lap)
        p[1] = (T)prm[0];             // L (pointwise)
    } else if (phys == PHIX_PHYS_CH) {
        p[0] = (T)prm[0];              // M
        p[1] = (T)(-prm[1]);           // -kappa
        p[2] = (T)2 * (T)prm[2];       // 2 rho
        p[3] = (T)prm[3];              // ca
        p[4] = (T)prm[4];              // cb
    } else {
        p[0] = (T)prm[0];              // M
        p[1] = (T)(-prm[2]);           // -kappa_c
        p[2] = (T)(prm[1] * prm[3]);   // L*kappa_eta
        p[3] = (T)(-prm[1]);           // -L
        p[4] = (T)2 * (T)prm[4];       // 2 lambda
    }
}
template void make_coeffs<float>(int, const double*, float*);
template void make_coeffs<double>(int, const double*, double*);

}  // namespace phix

using namespace phix;

// ---------------------------------------------------------------------------
// stepper object
// ---------------------------------------------------------------------------
struct phix_stepper {
    int phys = 0, scheme = 0, prec = 0, nf = 1, dim = 2;
    double prm[8] = {0};
    double dt = 0.0;
    phix_grid_t g{};
    Layout L{};        // the grid's stored layout (callers' arrays)
    Layout Lk{};       // layout of the stepper's own arrays (rows padded for 3-D FP32)
    size_t S = 0;      // stored elements per field (callers' arrays)
    size_t Sk = 0;     // elements per field of the stepper's own arrays
    size_t esz = 8;    // element size of the state
    void* st[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    void* lo[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // FP32: low parts of the state
    bool own_state = true;
    void* kbuf[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};
    int cur = 0;
    bool mu_zero_pending = false;  // MULTISTEP: the STEADY field is zeroed by its first evaluation
    // The first step of a loaded state applies every BC to the whole stored
    // arrays (as the reference's step does), which also fills the ghost cells
    // of padding planes; the fused kernels keep the physical plane's ghosts
    // current from then on.
    bool bc_pending = false;
    bool fuse_steps = true;  // one launch per RK4 step where step2d supports the grid (FP32 default)
    int tile = -1;           // 2-D stage tiles: -1 generic box tiles (fastest measured), else kColCfgs index
    cudaStream_t cap = nullptr;
    int graph_steps = 0;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    int graph_launches[2] = {0, 0};       // kernel launches recorded in each graph
    bool graph_flip[2] = {false, false};  // whether replaying it swaps the state buffers
    int* err = nullptr;            // device flag: a fused 3-D step gave up waiting for a plane copy
    bool fuse3d = true;            // 3-D RK4 of the mu physics: two launches of two fused stages
    double* stage_host = nullptr;  // device FP64 staging for run_host / diagnostics
    double* partials = nullptr;
    int partials_n = 0;
};

namespace phix {

// ---------------------------------------------------------------------------
// 3-D RK4 of the mu physics: two launches of two fused stages
// (march3d_fused.cuh), input planes by TMA
// ---------------------------------------------------------------------------
namespace {

// tiles (TX, TY, threads) of launch A (stages 1-2) and launch B (stages 3-4),
// two variants per precision (phix_stepper_set_tiles 0 / 1 on 3-D grids, -1 =
// 0).  Variant 0: the largest tiles (FP32 A 113 KB of shared memory, two CTAs
// per SM; B 173 KB, one); variant 1: B at 32x8 (FP32 113 KB, two CTAs per SM)
// and, in FP64, A at 32x8 too.
template <typename T, int V> struct M2Cfg;
template <> struct M2Cfg<float, 0> {
    static constexpr int AX = 32, AY = 16, ANT = 256, BX = 32, BY = 16, BNT = 512;
};
template <> struct M2Cfg<float, 1> {
    static constexpr int AX = 32, AY = 16, ANT = 256, BX = 32, BY = 8, BNT = 256;
};
template <> struct M2Cfg<double, 0> {
    static constexpr int AX = 32, AY = 16, ANT = 512, BX = 32, BY = 8, BNT = 512;
};
template <> struct M2Cfg<double, 1> {
    static constexpr int AX = 32, AY = 8, ANT = 256, BX = 32, BY = 8, BNT = 256;
};

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
        else
            cudaGetLastError();
    }
    return fn;
}

// Tensor map over a stored array of layout L (x, y, z = row, rows, planes;
// the padding columns of a row-padded layout are in bounds), boxes of
// WB x HB x 1 elements, no swizzle, zero fill outside.
int plane_map(CUtensorMap* m, const void* base, const Layout& L, int esz, int WB, int HB) {
    auto enc = tensor_map_encoder();
    if (!enc) { set_error("cuTensorMapEncodeTiled is not available"); return PHIX_ERR_UNSUPPORTED; }
    const int sy = L.s[2] / L.s[1], sz = L.n[2] + 2 * L.ghost;
    cuuint64_t dims[3] = {(cuuint64_t)L.s[1], (cuuint64_t)sy, (cuuint64_t)sz};
    cuuint64_t strides[2] = {(cuuint64_t)L.s[1] * esz, (cuuint64_t)L.s[2] * esz};
    cuuint32_t box[3] = {(cuuint32_t)WB, (cuuint32_t)HB, 1u};
    cuuint32_t estr[3] = {1u, 1u, 1u};
    const CUresult r = enc(m, esz == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
                           const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) { set_error("cuTensorMapEncodeTiled failed (%d)", (int)r); return PHIX_ERR_CUDA; }
    return PHIX_OK;
}

// Output planes per CTA: the z chunking of the tile columns that takes the
// fewest (waves x planes marched per CTA), a CTA marching rz + 2E planes.
int pick_rz(long long columns, int n2, int slots, int E) {
    int best_rz = n2;
    double best = 1e300;
    for (int nzc = 1; nzc <= (n2 + 7) / 8; ++nzc) {
        const int rz = (n2 + nzc - 1) / nzc;
        const long long ctas = columns * ((n2 + rz - 1) / rz);
        const long long waves = (ctas + slots - 1) / slots;
        const double cost = (double)waves * (rz + 2 * E);
        if (cost < best) { best = cost; best_rz = rz; }
    }
    return best_rz;
}

template <typename T, class Pol, int TX, int TY, int NT, bool B>
int m2_kernel(bool prepare, March2Args<T>* a, cudaStream_t s) {
    using G = March2<T, Pol, TX, TY, B>;
    static_assert(G::smem_bytes() <= 227 * 1024, "fused 3-D tile too large");
    auto kern = stage2_march3d<T, Pol, TX, TY, NT, B>;
    if (prepare) {
        PHIX_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::smem_bytes()));
        return PHIX_OK;
    }
    static int slots = 0;  // resident CTAs on the device
    if (!slots) {
        int dev = 0, nsm = 0, occ = 0;
        PHIX_TRY_CUDA(cudaGetDevice(&dev));
        PHIX_TRY_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        PHIX_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, NT, G::smem_bytes()));
        slots = (occ > 0 ? occ : 1) * nsm;
    }
    const Layout& L = a->S.L;
    int rc;
    for (int f = 0; f < G::NF; ++f) {
        if ((rc = plane_map(&a->tu[f], a->S.u[f], L, (int)sizeof(T), G::WB, G::HB))) return rc;
        if (B && (rc = plane_map(&a->tk[f], a->k2[f], L, (int)sizeof(T), G::WB, G::HB))) return rc;
    }
    const long long cols = (long long)((L.n[0] + TX - 1) / TX) * ((L.n[1] + TY - 1) / TY);
    a->rz = pick_rz(cols, L.n[2], slots, G::E);
    dim3 grid((L.n[0] + TX - 1) / TX, (L.n[1] + TY - 1) / TY, (L.n[2] + a->rz - 1) / a->rz);
    kern<<<grid, NT, G::smem_bytes(), s>>>(*a);
    PHIX_LAUNCH_CHECK(B ? "stage2_march3d(B)" : "stage2_march3d(A)");
    return PHIX_OK;
}

template <typename T, class Pol, int V>
int m2_step_v(bool prepare, March2Args<T>* a, cudaStream_t s, bool second) {
    using C = M2Cfg<T, V>;
    if (prepare) {
        int rc = m2_kernel<T, Pol, C::AX, C::AY, C::ANT, false>(true, nullptr, s);
        return rc ? rc : m2_kernel<T, Pol, C::BX, C::BY, C::BNT, true>(true, nullptr, s);
    }
    return second ? m2_kernel<T, Pol, C::BX, C::BY, C::BNT, true>(false, a, s)
                  : m2_kernel<T, Pol, C::AX, C::AY, C::ANT, false>(false, a, s);
}

// variant < 0: prepare every variant (prepare) or run variant 0
template <typename T, class Pol>
int m2_step(bool prepare, March2Args<T>* a, cudaStream_t s, bool second, int variant) {
    if (prepare) {
        int rc = m2_step_v<T, Pol, 0>(true, a, s, second);
        return rc ? rc : m2_step_v<T, Pol, 1>(true, a, s, second);
    }
    return variant == 1 ? m2_step_v<T, Pol, 1>(false, a, s, second) : m2_step_v<T, Pol, 0>(false, a, s, second);
}

template <typename T>
int m2_dispatch(int phys, bool prepare, March2Args<T>* a, cudaStream_t s, bool second, int variant = 0) {
    if (variant > 1) {
        set_error("fused 3-D step: tile variant %d (0 or 1)", variant);
        return PHIX_ERR_UNSUPPORTED;
    }
    if (phys == PHIX_PHYS_CH) return m2_step<T, PolCH>(prepare, a, s, second, variant);
    if (phys == PHIX_PHYS_CHAC) return m2_step<T, PolCHAC>(prepare, a, s, second, variant);
    set_error("fused 3-D step: physics %d has no chemical potential", phys);
    return PHIX_ERR_UNSUPPORTED;
}

// ---- one stage of the mu physics streamed through z (stream3d.cuh) --------
// tile variants per precision: TX x TY tile, R rows of a column per thread,
// (TX + 4) x (TY + 4) / R threads; variant 0 is the default (measured fastest
// at 256^3: FP32 32x8, FP64 32x6, whose k stages fit three CTAs per SM)
constexpr int kNumS3Variants = 3;
template <typename T, int V> struct S3Cfg;
template <> struct S3Cfg<float, 0> { static constexpr int TX = 32, TY = 8, R = 1; };
template <> struct S3Cfg<float, 1> { static constexpr int TX = 32, TY = 16, R = 4; };
template <> struct S3Cfg<float, 2> { static constexpr int TX = 32, TY = 6, R = 1; };
template <> struct S3Cfg<double, 0> { static constexpr int TX = 32, TY = 6, R = 1; };
template <> struct S3Cfg<double, 1> { static constexpr int TX = 32, TY = 8, R = 2; };
template <> struct S3Cfg<double, 2> { static constexpr int TX = 32, TY = 8, R = 1; };

template <typename T, class Pol, int MODE, int V>
int s3_kernel(bool prepare, Stream3Args<T>* a, cudaStream_t s) {
    using C = S3Cfg<T, V>;
    using G = Stream3<T, Pol, C::TX, C::TY, C::R, MODE != MODE_K>;
    static_assert(G::smem_bytes() <= 227 * 1024, "streamed 3-D tile too large");
    auto kern = stage_stream3d<T, Pol, MODE, C::TX, C::TY, C::R>;
    if (prepare) {
        PHIX_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::smem_bytes()));
        return PHIX_OK;
    }
    static int slots = 0;  // resident CTAs on the device
    if (!slots) {
        int dev = 0, nsm = 0, occ = 0;
        PHIX_TRY_CUDA(cudaGetDevice(&dev));
        PHIX_TRY_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        PHIX_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, G::NT, G::smem_bytes()));
        slots = (occ > 0 ? occ : 1) * nsm;
    }
    const Layout& L = a->S.L;
    int rc;
    for (int f = 0; f < G::NF; ++f) {
        if ((rc = plane_map(&a->tu[f], a->S.u[f], L, (int)sizeof(T), G::WB, G::HB))) return rc;
        if (a->S.kin[0] && (rc = plane_map(&a->tk[f], a->S.kin[f], L, (int)sizeof(T), G::WB, G::HB))) return rc;
    }
    a->pfm = 0;
    if (MODE != MODE_K && sizeof(T) == 8) {
        // L2 prefetch boxes of the update's other operands (16-byte aligned arrays only)
        for (int f = 0; f < G::NF; ++f) {
            const void* src[3] = {MODE == MODE_RK4_FINAL ? a->S.k1[f] : nullptr,
                                  MODE == MODE_RK4_FINAL ? a->S.k2[f] : nullptr, a->S.ulo[f]};
            for (int j = 0; j < 3; ++j) {
                if (!src[j] || (uintptr_t)src[j] % 16 != 0) continue;
                if ((rc = plane_map(&a->tq[j][f], src[j], L, (int)sizeof(T), C::TX + G::VEC, C::TY))) return rc;
                a->pfm |= 1 << (2 * j + f);
            }
        }
    }
    const long long cols = (long long)((L.n[0] + C::TX - 1) / C::TX) * ((L.n[1] + C::TY - 1) / C::TY);
    a->rz = pick_rz(cols, L.n[2], slots, G::H);
    dim3 grid((L.n[0] + C::TX - 1) / C::TX, (L.n[1] + C::TY - 1) / C::TY, (L.n[2] + a->rz - 1) / a->rz);
    kern<<<grid, G::NT, G::smem_bytes(), s>>>(*a);
    PHIX_LAUNCH_CHECK("stage_stream3d");
    return PHIX_OK;
}

template <typename T, class Pol, int V>
int s3_mode_v(int mode, bool prepare, Stream3Args<T>* a, cudaStream_t s) {
    if (prepare) {
        int rc = s3_kernel<T, Pol, MODE_K, V>(true, a, s);
        if (!rc) rc = s3_kernel<T, Pol, MODE_RK4_FINAL, V>(true, a, s);
        return rc ? rc : s3_kernel<T, Pol, MODE_EULER_FINAL, V>(true, a, s);
    }
    switch (mode) {
        case MODE_K: return s3_kernel<T, Pol, MODE_K, V>(false, a, s);
        case MODE_RK4_FINAL: return s3_kernel<T, Pol, MODE_RK4_FINAL, V>(false, a, s);
        case MODE_EULER_FINAL: return s3_kernel<T, Pol, MODE_EULER_FINAL, V>(false, a, s);
    }
    set_error("stage_stream3d: mode %d", mode);
    return PHIX_ERR_UNSUPPORTED;
}

// prepare: every variant; else the one asked for
template <typename T, class Pol>
int s3_mode(int mode, bool prepare, Stream3Args<T>* a, cudaStream_t s, int variant) {
    if (prepare) {
        int rc = s3_mode_v<T, Pol, 0>(mode, true, a, s);
        if (!rc) rc = s3_mode_v<T, Pol, 1>(mode, true, a, s);
        return rc ? rc : s3_mode_v<T, Pol, 2>(mode, true, a, s);
    }
    switch (variant) {
        case 0: return s3_mode_v<T, Pol, 0>(mode, false, a, s);
        case 1: return s3_mode_v<T, Pol, 1>(mode, false, a, s);
        case 2: return s3_mode_v<T, Pol, 2>(mode, false, a, s);
    }
    set_error("stage_stream3d: tile variant %d (0..%d)", variant, kNumS3Variants - 1);
    return PHIX_ERR_UNSUPPORTED;
}

template <typename T>
int s3_dispatch(int phys, int mode, bool prepare, Stream3Args<T>* a, cudaStream_t s, int variant = 0) {
    if (phys == PHIX_PHYS_CH) return s3_mode<T, PolCH>(mode, prepare, a, s, variant);
    if (phys == PHIX_PHYS_CHAC) return s3_mode<T, PolCHAC>(mode, prepare, a, s, variant);
    set_error("stage_stream3d: physics %d has no chemical potential", phys);
    return PHIX_ERR_UNSUPPORTED;
}

}  // namespace

// The 3-D stage kernels with TMA plane staging take the grid: CH or CH+AC,
// z periodic, x and y periodic or zero-flux, rows of whole 16-byte units,
// 16-byte aligned arrays (the stepper's own arrays are row-padded).
static bool tma3d_ok(const phix_stepper* h) {
    if (h->dim != 3 || (h->phys != PHIX_PHYS_CH && h->phys != PHIX_PHYS_CHAC)) return false;
    const Layout& L = h->Lk;
    for (int i = 0; i < 4; ++i)
        if (L.bc[i] != PHIX_BC_PERIODIC && L.bc[i] != PHIX_BC_NOFLUX) return false;
    if (L.bc[4] != PHIX_BC_PERIODIC) return false;
    if ((L.s[1] * h->esz) % 16 != 0) return false;
    for (int f = 0; f < h->nf; ++f)
        for (int b = 0; b < 2; ++b)
            if ((uintptr_t)h->st[b][f] % 16 != 0) return false;
    return tensor_map_encoder() != nullptr;
}

// Tile configuration of 3-D steppers that selects the marching stage kernel
// (no TMA) for one launch per stage.
constexpr int TILE3D_MARCH = 2;
// Tile configurations 3 .. 3 + kNumS3Variants - 1 of 3-D steppers: the
// streamed stage kernel's tile variants (-1, 0 and 1: variant 0).
constexpr int TILE3D_STREAM = 3;

// One 3-D stage: streamed with TMA staging where tma3d_ok (unless the tile
// configuration asks for the marching kernel), else stage_march3d.
template <typename T>
static int launch_stage3d(const phix_stepper* h, int mode, const StageArgs<T>& A, cudaStream_t s) {
    if (h->dim == 3 && h->tile != TILE3D_MARCH && tma3d_ok(h)) {
        Stream3Args<T> a;
        memset(&a, 0, sizeof(a));
        a.S = A;
        a.err = h->err;
        const int v = h->tile >= TILE3D_STREAM && h->tile < TILE3D_STREAM + kNumS3Variants ? h->tile - TILE3D_STREAM : 0;
        return s3_dispatch<T>(h->phys, mode, false, &a, s, v);
    }
    return launch_stage<T>(h->phys, h->dim, mode, A, s, h->tile);
}

// The fused 3-D path takes the grid: RK4 of CH or CH+AC, z periodic, x and y
// periodic or zero-flux, rows of whole 16-byte units, 16-byte aligned arrays.
static bool step3d_fused(const phix_stepper* h) {
    return h->fuse_steps && h->fuse3d && h->scheme == PHIX_RK4 && tma3d_ok(h);
}

static void drop_graphs(phix_stepper* h) {
    for (auto& e : h->gexec)
        if (e) { cudaGraphExecDestroy(e); e = nullptr; }
}

static bool step_fused(const phix_stepper* h) {
    return h->fuse_steps && h->scheme == PHIX_RK4 && h->nf == 1 && step2d_supported(h->L, h->dim);
}

// Multi-step steppers on 2-D grids with four periodic sides run the pair
// kernel unless one launch per step is switched off (then stage_box).
static bool ms_pair(const phix_stepper* h) {
    return h->fuse_steps && h->scheme == PHIX_MULTISTEP && h->dim == 2 && step_pair_supported(h->L, 2);
}

static int launches_per_step(const phix_stepper* h) {
    if (step3d_fused(h)) return 2;
    return h->scheme == PHIX_RK4 && !step_fused(h) ? 4 : 1;
}

template <typename T>
static int enqueue_step(phix_stepper* h, cudaStream_t s, int depth) {
    StageArgs<T> A;
    memset(&A, 0, sizeof(A));
    A.L = h->Lk;
    for (int a = 0; a < 3; ++a) A.i2[a] = a < h->dim ? (T)(1.0 / (h->g.d[a] * h->g.d[a])) : (T)0;
    make_coeffs<T>(h->phys, h->prm, A.p);
    const int c = h->cur, o = 1 - c;
    for (int f = 0; f < h->nf; ++f) A.u[f] = (const T*)h->st[c][f];
    // compensated FP32 state: the final stage reads lo[c] and writes lo[o]
    auto set_lo = [&](int nfl) {
        for (int f = 0; f < nfl; ++f)
            if (h->lo[c][f]) {
                A.ulo[f] = (const T*)h->lo[c][f];
                A.outlo[f] = (T*)h->lo[o][f];
            }
    };
    int rc;
    if (h->scheme == PHIX_MULTISTEP) {
        A.u[1] = nullptr;
        A.out[0] = (T*)h->st[o][0];
        A.mu_out = (T*)h->st[0][1];
        A.dtf = (T)h->dt;
        set_lo(1);
        rc = ms_pair(h) ? launch_ms<T>(A, s, h->tile) : launch_stage<T>(h->phys, h->dim, MODE_MULTISTEP, A, s, h->tile);
        if (rc) return rc;
    } else if (h->scheme == PHIX_EULER) {
        for (int f = 0; f < h->nf; ++f) A.out[f] = (T*)h->st[o][f];
        A.dtf = (T)h->dt;
        set_lo(h->nf);
        rc = launch_stage3d<T>(h, MODE_EULER_FINAL, A, s);
        if (rc) return rc;
    } else if (step_fused(h)) {
        A.out[0] = (T*)h->st[o][0];
        A.dtf = (T)(h->dt / 6.0);
        set_lo(1);
        StepArgs<T> B;
        B.S = A;
        B.dt2 = (T)(h->dt * 0.5);
        B.dt = (T)h->dt;
        if ((rc = launch_step2d<T>(h->phys, B, s, h->tile, depth))) return rc;
    } else if (step3d_fused(h)) {
        // launch A: k2 and acc = k1 + 2 k2; launch B: the new state
        const T dt2 = (T)(h->dt * 0.5), dtt = (T)h->dt;
        for (int f = 0; f < h->nf; ++f) A.out[f] = (T*)h->st[o][f];
        A.dtf = (T)(h->dt / 6.0);
        set_lo(h->nf);
        March2Args<T> M;
        memset(&M, 0, sizeof(M));
        M.S = A;
        for (int f = 0; f < h->nf; ++f) {
            M.k2[f] = (T*)h->kbuf[1][f];
            M.acc[f] = (T*)h->kbuf[0][f];
        }
        M.err = h->err;
        M.a_in = dt2;
        M.a_mid = dt2;
        if ((rc = m2_dispatch<T>(h->phys, false, &M, s, false, h->tile))) return rc;
        M.a_mid = dtt;
        if ((rc = m2_dispatch<T>(h->phys, false, &M, s, true, h->tile))) return rc;
    } else {
        const T dt2 = (T)(h->dt * 0.5), dtt = (T)h->dt;
        // stage 1
        for (int f = 0; f < h->nf; ++f) A.out[f] = (T*)h->kbuf[0][f];
        if ((rc = launch_stage3d<T>(h, MODE_K, A, s))) return rc;
        // stages 2, 3
        for (int st = 1; st < 3; ++st) {
            for (int f = 0; f < h->nf; ++f) {
                A.kin[f] = (const T*)h->kbuf[st - 1][f];
                A.out[f] = (T*)h->kbuf[st][f];
            }
            A.a = dt2;
            if ((rc = launch_stage3d<T>(h, MODE_K, A, s))) return rc;
        }
        // stage 4 + update
        for (int f = 0; f < h->nf; ++f) {
            A.kin[f] = (const T*)h->kbuf[2][f];
            A.k1[f] = (const T*)h->kbuf[0][f];
            A.k2[f] = (const T*)h->kbuf[1][f];
            A.out[f] = (T*)h->st[o][f];
        }
        A.a = dtt;
        A.dtf = (T)(h->dt / 6.0);
        set_lo(h->nf);
        if ((rc = launch_stage3d<T>(h, MODE_RK4_FINAL, A, s))) return rc;
    }
    h->cur = o;
    return PHIX_OK;
}

// Time steps per launch of the current settings: 2 for a temporally blocked
// pair tile (an odd remainder of steps runs as one single-step launch).
static int step_depth(const phix_stepper* h) { return step_fused(h) ? step_cfg_depth(h->tile) : 1; }

static int enqueue_steps(phix_stepper* h, int n, cudaStream_t s, int* launches = nullptr) {
    const int d = step_depth(h);
    for (int i = 0; i < n;) {
        const int k = d == 2 && n - i >= 2 ? 2 : 1;
        int rc = h->prec == PHIX_F32 ? enqueue_step<float>(h, s, k) : enqueue_step<double>(h, s, k);
        if (rc) return rc;
        if (launches) *launches += launches_per_step(h);
        i += k;
    }
    return PHIX_OK;
}

static int replay_group(phix_stepper* h, cudaStream_t s) {
    const int parity = h->cur;
    if (!h->gexec[parity]) {
        cudaGraph_t graph = nullptr;
        PHIX_TRY_CUDA(cudaStreamBeginCapture(h->cap, cudaStreamCaptureModeThreadLocal));
        int rc, launches = 0;
        {
            LaunchCountPause pause;  // recorded, not launched: the replay below counts them
            rc = enqueue_steps(h, h->graph_steps, h->cap, &launches);
        }
        cudaError_t e = cudaStreamEndCapture(h->cap, &graph);
        h->graph_flip[parity] = h->cur != parity;  // each launch swaps the state buffers
        h->graph_launches[parity] = launches;
        if (rc) { if (graph) cudaGraphDestroy(graph); h->cur = parity; return rc; }
        if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&h->gexec[parity], graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return cuda_status(e, "cudaGraphInstantiate");
        h->cur = parity;  // capture only recorded; the replay below advances
    }
    PHIX_TRY_CUDA(cudaGraphLaunch(h->gexec[parity], s));
    // launches inside the graph count as kernel launches of this library
    count_launch(h->graph_launches[parity]);
    if (h->graph_flip[parity]) h->cur = 1 - parity;
    return PHIX_OK;
}

}  // namespace phix

extern "C" {

int phix_stepper_create(phix_stepper_t** out, int phys, int scheme, int precision, const double* prm, double dt,
                        const phix_grid_t* g) {
    if (!out) { set_error("out is NULL"); return PHIX_ERR_ARG; }
    *out = nullptr;
    if (physics_nfields(phys) == 0) { set_error("unknown physics %d", phys); return PHIX_ERR_ARG; }
    if (scheme != PHIX_EULER && scheme != PHIX_RK4 && scheme != PHIX_MULTISTEP) {
        set_error("unknown scheme %d", scheme);
        return PHIX_ERR_ARG;
    }
    if (precision != PHIX_F32 && precision != PHIX_F64) { set_error("unknown precision %d", precision); return PHIX_ERR_ARG; }
    if (!prm) { set_error("prm is NULL"); return PHIX_ERR_ARG; }
    Layout L;
    size_t S;
    int rc = validate_grid(g, &L, &S);
    if (rc) return rc;
    if (scheme == PHIX_MULTISTEP && (phys != PHIX_PHYS_CH || g->dim > 2 || g->ghost != 1)) {
        set_error("multi-step scheme: Cahn-Hilliard on 1-D/2-D grids with ghost 1 only");
        return PHIX_ERR_UNSUPPORTED;
    }
    auto* h = new (std::nothrow) phix_stepper();
    if (!h) { set_error("out of host memory"); return PHIX_ERR_ARG; }
    h->phys = phys;
    h->scheme = scheme;
    h->prec = precision;
    h->nf = scheme == PHIX_MULTISTEP ? 2 : physics_nfields(phys);
    h->dim = g->dim;
    memcpy(h->prm, prm, sizeof(double) * (phys == PHIX_PHYS_AC ? 2 : 5));
    h->dt = dt;
    h->g = *g;
    h->L = L;
    h->S = S;
    h->esz = precision == PHIX_F32 ? 4 : 8;
    // 3-D steppers keep their own arrays with rows padded to whole 16-byte
    // units (a TMA row stride must be one); the ghost layers stay where the
    // layout's origin puts them, the padding columns are never read
    h->Lk = L;
    h->Sk = S;
    if (g->dim == 3) {
        const int vec = 16 / (int)h->esz;
        const int sx = L.s[1], pk = (sx + vec - 1) / vec * vec, sy = L.s[2] / L.s[1], gh = L.ghost;
        h->Lk.s[1] = pk;
        h->Lk.s[2] = pk * sy;
        h->Lk.origin = gh + pk * (gh + sy * gh);
        h->Sk = (size_t)pk * sy * (L.n[2] + 2 * gh);
    }
    // measured on B200 at 1024^2: the one-launch step wins in FP32, and in FP64
    // where the pair kernel takes the grid (CH, four periodic sides); the
    // cell-per-thread step kernel loses to one launch per stage in FP64
    // 3-D: one launch per stage by default (measured faster on B200 than the
    // fused two-stage launches, which the autotuner may still pick)
    h->fuse_steps = g->dim < 3 && (precision == PHIX_F32 || (phys == PHIX_PHYS_CH && step_pair_supported(L, g->dim)));
    auto fail = [&](cudaError_t e, const char* w) {
        int r = cuda_status(e, w);
        phix_stepper_destroy(h);
        return r;
    };
    cudaError_t e;
    for (int b = 0; b < 2; ++b)
        for (int f = 0; f < h->nf; ++f) {
            if ((e = cudaMalloc(&h->st[b][f], h->Sk * h->esz)) != cudaSuccess) return fail(e, "cudaMalloc(state)");
            if ((e = cudaMemset(h->st[b][f], 0, h->Sk * h->esz)) != cudaSuccess) return fail(e, "cudaMemset(state)");
        }
    if (precision == PHIX_F32) {
        // the multi-step mu is recomputed every step: no low part
        const int nlo = scheme == PHIX_MULTISTEP ? 1 : h->nf;
        for (int b = 0; b < 2; ++b)
            for (int f = 0; f < nlo; ++f) {
                if ((e = cudaMalloc(&h->lo[b][f], h->Sk * 4)) != cudaSuccess) return fail(e, "cudaMalloc(lo)");
                if ((e = cudaMemset(h->lo[b][f], 0, h->Sk * 4)) != cudaSuccess) return fail(e, "cudaMemset(lo)");
            }
    }
    if (scheme == PHIX_RK4)
        for (int k = 0; k < 3; ++k)
            for (int f = 0; f < h->nf; ++f) {
                // ghosts of k stay zero: kernels only ever write physical cells
                if ((e = cudaMalloc(&h->kbuf[k][f], h->Sk * h->esz)) != cudaSuccess) return fail(e, "cudaMalloc(k)");
                if ((e = cudaMemset(h->kbuf[k][f], 0, h->Sk * h->esz)) != cudaSuccess) return fail(e, "cudaMemset(k)");
            }
    if ((e = cudaMalloc(&h->err, sizeof(int))) != cudaSuccess) return fail(e, "cudaMalloc(err)");
    if ((e = cudaMemset(h->err, 0, sizeof(int))) != cudaSuccess) return fail(e, "cudaMemset(err)");
    if ((e = cudaStreamCreateWithFlags(&h->cap, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "cudaStreamCreate");
    if ((rc = prepare_stage(phys, g->dim, precision))) {
        phix_stepper_destroy(h);
        return rc;
    }
    if (g->dim == 3 && scheme != PHIX_MULTISTEP && phys != PHIX_PHYS_AC) {
        rc = precision == PHIX_F32 ? s3_dispatch<float>(phys, 0, true, nullptr, 0)
                                   : s3_dispatch<double>(phys, 0, true, nullptr, 0);
        if (rc) {
            phix_stepper_destroy(h);
            return rc;
        }
    }
    if (g->dim == 3 && scheme == PHIX_RK4 && phys != PHIX_PHYS_AC) {
        rc = precision == PHIX_F32 ? m2_dispatch<float>(phys, true, nullptr, 0, false)
                                   : m2_dispatch<double>(phys, true, nullptr, 0, false);
        if (rc) {
            phix_stepper_destroy(h);
            return rc;
        }
    }
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return fail(e, "cudaDeviceSynchronize");
    *out = h;
    return PHIX_OK;
}

int phix_stepper_destroy(phix_stepper_t* h) {
    if (!h) return PHIX_OK;
    drop_graphs(h);
    if (h->own_state)
        for (auto& b : h->st)
            for (auto& p : b)
                if (p) cudaFree(p);
    for (auto& k : h->kbuf)
        for (auto& p : k)
            if (p) cudaFree(p);
    for (auto& b : h->lo)
        for (auto& p : b)
            if (p) cudaFree(p);
    if (h->stage_host) cudaFree(h->stage_host);
    if (h->partials) cudaFree(h->partials);
    if (h->err) cudaFree(h->err);
    if (h->cap) cudaStreamDestroy(h->cap);
    delete h;
    return PHIX_OK;
}

int phix_stepper_nfields(const phix_stepper_t* h) { return h ? h->nf : 0; }

int phix_stepper_current(const phix_stepper_t* h) { return h ? h->cur : -1; }

int phix_stepper_set_graph(phix_stepper_t* h, int steps_per_graph) {
    if (!h || steps_per_graph < 0) { set_error("bad stepper or steps_per_graph"); return PHIX_ERR_ARG; }
    drop_graphs(h);
    h->graph_steps = steps_per_graph;
    return PHIX_OK;
}

int phix_stepper_set_fusion(phix_stepper_t* h, int one_launch_per_step) {
    if (!h) { set_error("set_fusion: NULL stepper"); return PHIX_ERR_ARG; }
    const bool f = one_launch_per_step != 0;
    if (f != h->fuse_steps) {
        drop_graphs(h);
        h->fuse_steps = f;
    }
    return PHIX_OK;
}

int phix_stepper_launches_per_step(const phix_stepper_t* h) { return h ? launches_per_step(h) : -1; }

int phix_stepper_depth(const phix_stepper_t* h) { return h ? step_depth(h) : -1; }

int phix_stepper_set_tiles(phix_stepper_t* h, int tile_cfg) {
    if (!h || tile_cfg < -1 || tile_cfg >= (kNumColCfgs > kNumStepCfgs + kNumPairCfgs ? kNumColCfgs
                                                                                       : kNumStepCfgs + kNumPairCfgs)) {
        set_error("set_tiles: bad stepper or configuration");
        return PHIX_ERR_ARG;
    }
    if (tile_cfg != h->tile) {
        drop_graphs(h);
        h->tile = tile_cfg;
    }
    return PHIX_OK;
}

int phix_stepper_get_tiles(const phix_stepper_t* h, int* one_launch_per_step, int* tile_cfg) {
    if (!h) { set_error("get_tiles: NULL stepper"); return PHIX_ERR_ARG; }
    if (one_launch_per_step) *one_launch_per_step = step_fused(h) || ms_pair(h) ? 1 : 0;
    if (tile_cfg) *tile_cfg = h->tile;
    return PHIX_OK;
}

int phix_stepper_autotune(phix_stepper_t* h, int trial_steps, double* best_ms) {
    if (!h || trial_steps < 1) { set_error("autotune: bad stepper or trial_steps"); return PHIX_ERR_ARG; }
    // candidates: one launch per stage with every stage tile, and (RK4, one
    // 2-D field with periodic or zero-flux sides) one launch per step with
    // every step tile; multi-step: stage_box, and the pair kernel with every
    // tile where the grid takes it
    std::vector<std::pair<bool, int>> cand;
    if (h->scheme == PHIX_MULTISTEP) {
        cand.push_back({false, -1});
        if (h->dim == 2 && step_pair_supported(h->L, 2))
            for (int t = 0; t < kNumMsCfgs; ++t) cand.push_back({true, t});
    } else {
        if (h->dim == 2)
            for (int t = -1; t < kNumColCfgs; ++t) cand.push_back({false, t});
        else
            cand.push_back({false, -1});
        if (h->dim == 3) {
            cand.push_back({false, TILE3D_MARCH});  // the marching stage kernel
            for (int v = 1; v < kNumS3Variants; ++v) cand.push_back({false, TILE3D_STREAM + v});  // streamed variants
        }
        if (h->dim == 3 && h->scheme == PHIX_RK4 && h->phys != PHIX_PHYS_AC) {
            cand.push_back({true, 0});  // the fused two-stage tile variants
            cand.push_back({true, 1});
        }
        if (h->scheme == PHIX_RK4 && h->nf == 1 && step2d_supported(h->L, h->dim))
            for (int t = 0; t < kNumStepCfgs + kNumPairCfgs; ++t) cand.push_back({true, t});
    }

    // trials advance the state: save it, and restore it afterwards
    const int cur0 = h->cur;
    const bool bc0 = h->bc_pending, fuse0 = h->fuse_steps;
    const int tile0 = h->tile, graph0 = h->graph_steps;
    const size_t bytes = h->Sk * h->esz;
    const int parts = h->lo[cur0][0] ? 2 : 1;
    void* save = nullptr;
    PHIX_TRY_CUDA(cudaMalloc(&save, bytes * h->nf * parts));
    // the multi-step mu field is one buffer (st[0][1]) with no low part
    const bool ms = h->scheme == PHIX_MULTISTEP;
    auto copy_state = [&](bool to_save) {
        for (int f = 0; f < h->nf; ++f)
            for (int q = 0; q < parts; ++q) {
                if (ms && f == 1 && q) continue;
                void* buf = q ? h->lo[cur0][f] : (ms && f == 1 ? h->st[0][1] : h->st[cur0][f]);
                char* sv = (char*)save + bytes * (f * parts + q);
                cudaError_t e = to_save ? cudaMemcpy(sv, buf, bytes, cudaMemcpyDeviceToDevice)
                                        : cudaMemcpy(buf, sv, bytes, cudaMemcpyDeviceToDevice);
                if (e != cudaSuccess) return cuda_status(e, "autotune: state copy");
            }
        return (int)PHIX_OK;
    };
    int rc = copy_state(true);
    drop_graphs(h);
    h->graph_steps = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (!rc && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
        rc = cuda_status(cudaGetLastError(), "autotune: cudaEventCreate");
    float best = 1e30f;
    bool best_fuse = fuse0;
    int best_tile = tile0;
    for (size_t c = 0; c < cand.size() && !rc; ++c) {
        h->fuse_steps = cand[c].first;
        h->tile = cand[c].second;
        int r = enqueue_steps(h, step_depth(h), 0);  // warm-up; shapes this grid cannot take are skipped
        if (r == PHIX_ERR_UNSUPPORTED) continue;
        if (r) { rc = r; break; }
        float ms = 1e30f;
        for (int rep = 0; rep < 2 && !rc; ++rep) {  // the faster of two timings
            cudaEventRecord(e0, 0);
            if ((rc = enqueue_steps(h, trial_steps, 0))) break;
            cudaEventRecord(e1, 0);
            cudaError_t e = cudaEventSynchronize(e1);
            if (e != cudaSuccess) { rc = cuda_status(e, "autotune: trial"); break; }
            float t = 0.f;
            cudaEventElapsedTime(&t, e0, e1);
            ms = std::min(ms, t);
        }
        if (rc) break;
        if (ms < best) { best = ms; best_fuse = cand[c].first; best_tile = cand[c].second; }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    h->cur = cur0;
    const int rc2 = copy_state(false);
    cudaFree(save);
    h->bc_pending = bc0;
    h->graph_steps = graph0;
    h->fuse_steps = rc ? fuse0 : best_fuse;
    h->tile = rc ? tile0 : best_tile;
    if (rc) return rc;
    if (rc2) return rc2;
    if (best_ms) *best_ms = best / trial_steps;
    return PHIX_OK;
}

int phix_stepper_bind(phix_stepper_t* h, double* const* fields, double* const* alt) {
    if (!h || !fields || !alt) { set_error("bind: NULL argument"); return PHIX_ERR_ARG; }
    if (h->prec != PHIX_F64) { set_error("bind: only FP64 steppers run on caller buffers"); return PHIX_ERR_UNSUPPORTED; }
    for (int f = 0; f < h->nf; ++f) {
        const bool single = h->scheme == PHIX_MULTISTEP && f == 1;  // mu: one buffer
        if (!fields[f] || (!single && (!alt[f] || fields[f] == alt[f]))) {
            set_error("bind: field %d buffers invalid", f);
            return PHIX_ERR_ARG;
        }
    }
    drop_graphs(h);
    if (h->own_state)
        for (auto& b : h->st)
            for (auto& p : b)
                if (p) { cudaFree(p); p = nullptr; }
    h->own_state = false;
    h->Lk = h->L;  // the callers' arrays have the grid's own layout (k buffers are large enough for it)
    for (int f = 0; f < h->nf; ++f) {
        h->st[0][f] = fields[f];
        h->st[1][f] = alt[f] ? alt[f] : fields[f];
    }
    h->cur = 0;
    h->mu_zero_pending = h->scheme == PHIX_MULTISTEP;
    h->bc_pending = true;
    return PHIX_OK;
}

int phix_stepper_status(phix_stepper_t* h, void* stream) {
    if (!h) { set_error("status: NULL stepper"); return PHIX_ERR_ARG; }
    cudaStream_t s = (cudaStream_t)stream;
    int herr = 0;
    PHIX_TRY_CUDA(cudaMemcpyAsync(&herr, h->err, sizeof(int), cudaMemcpyDeviceToHost, s));
    PHIX_TRY_CUDA(cudaMemsetAsync(h->err, 0, sizeof(int), s));
    PHIX_TRY_CUDA(cudaStreamSynchronize(s));
    if (herr) { set_error("stepper: a fused 3-D step gave up waiting for a plane copy"); return PHIX_ERR_TIMEOUT; }
    return PHIX_OK;
}

int phix_stepper_advance(phix_stepper_t* h, int nsteps, void* stream) {
    if (!h || nsteps < 0) { set_error("advance: bad stepper or nsteps"); return PHIX_ERR_ARG; }
    if (!h->st[0][0]) { set_error("advance: stepper has no state buffers"); return PHIX_ERR_ARG; }
    cudaStream_t s = (cudaStream_t)stream;
    int rc;
    if (h->mu_zero_pending && nsteps > 0) {
        PHIX_TRY_CUDA(cudaMemsetAsync(h->st[0][1], 0, h->S * h->esz, s));
        h->mu_zero_pending = false;
    }
    if (h->bc_pending && nsteps > 0) {
        for (int f = 0; f < h->nf; ++f)
            for (int b = 0; b < (h->scheme == PHIX_MULTISTEP && f == 1 ? 1 : 2); ++b) {  // one mu buffer
                if (h->prec == PHIX_F64) rc = bc_fill_layout<double>((double*)h->st[b][f], &h->g, h->Lk, false, s);
                else rc = bc_fill_layout<float>((float*)h->st[b][f], &h->g, h->Lk, false, s);
                if (rc) return rc;
                if (h->lo[b][f] && (rc = bc_fill_layout<float>((float*)h->lo[b][f], &h->g, h->Lk, true, s))) return rc;
            }
        h->bc_pending = false;
    }
    if (h->graph_steps > 0) {
        while (nsteps >= h->graph_steps) {
            if ((rc = replay_group(h, s))) return rc;
            nsteps -= h->graph_steps;
        }
    }
    return enqueue_steps(h, nsteps, s);
}

}  // extern "C"

// state conversion lives in convert.cu (needs a kernel)
namespace phix {
int stepper_copy_in(phix_stepper* h, const double* const* fields, cudaStream_t s);
int stepper_copy_out(phix_stepper* h, double* const* fields, cudaStream_t s);
int stepper_diag(phix_stepper* h, double* out);
void* stepper_state(phix_stepper* h, int f) {
    if (h->scheme == PHIX_MULTISTEP && f == 1) return h->st[0][1];  // single mu buffer
    return h->st[h->cur][f];
}
int stepper_scheme(const phix_stepper* h) { return h->scheme; }
void stepper_mark_loaded(phix_stepper* h) {
    h->mu_zero_pending = h->scheme == PHIX_MULTISTEP;
    h->bc_pending = true;
}
void* stepper_state_buf(phix_stepper* h, int b, int f) { return h->st[b][f]; }
void* stepper_lo_buf(phix_stepper* h, int b, int f) { return h->lo[b][f]; }
int stepper_cur(const phix_stepper* h) { return h->cur; }
size_t stepper_stored(const phix_stepper* h) { return h->S; }
const Layout& stepper_layout(const phix_stepper* h) { return h->Lk; }
const Layout& stepper_grid_layout(const phix_stepper* h) { return h->L; }
int stepper_prec(const phix_stepper* h) { return h->prec; }
int stepper_nf(const phix_stepper* h) { return h->nf; }
int stepper_phys(const phix_stepper* h) { return h->phys; }
const phix_grid_t* stepper_grid(const phix_stepper* h) { return &h->g; }
const double* stepper_prm(const phix_stepper* h) { return h->prm; }
double* stepper_staging(phix_stepper* h) {
    if (!h->stage_host) {
        if (cudaMalloc(&h->stage_host, h->S * sizeof(double) * h->nf) != cudaSuccess) return nullptr;
    }
    return h->stage_host;
}
double* stepper_partials(phix_stepper* h, int n) {
    if (h->partials_n < n) {
        if (h->partials) cudaFree(h->partials);
        h->partials = nullptr;
        h->partials_n = 0;
        if (cudaMalloc(&h->partials, sizeof(double) * n) != cudaSuccess) return nullptr;
        h->partials_n = n;
    }
    return h->partials;
}
}  // namespace phix
