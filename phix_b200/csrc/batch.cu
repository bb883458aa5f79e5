// batch.cu -- many independent simulations of uneven grid sizes and
// parameters in one persistent launch per RK stage (phix_batch_*).
//
// All instances share physics, scheme, precision and dim (2-D), and advance in
// lockstep.  Each has its own stored layout, BCs, coefficients, two state
// buffers and k1..k3, carved from one device pool.  A stage launch is one
// persistent kernel (stage_box_batched) over a tile list covering every
// instance (largest instances first), with per-instance StageArgs prepared
// once on the host for each (stage, parity) pair.  Groups of steps are
// captured into a CUDA graph.  The tile shape and the number of resident CTAs
// per SM are chosen by a measuring autotuner (phix_batch_autotune).
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "phix/detail/common.cuh"
#include "phix/detail/stage.cuh"
#include "phix/detail/step2d.cuh"
#include "phix/detail/step2d_pair.cuh"
#include "stepper.h"

namespace phix {
namespace {

struct TileCfg {
    int tx, ty, nt;
};
// Candidate tile shapes (index = PHIX tile config id).
constexpr TileCfg kTileCfgs[] = {{64, 16, 256}, {32, 16, 256}, {128, 8, 256}, {64, 8, 256}, {32, 32, 256}, {128, 16, 256}};
constexpr int kNumTileCfgs = sizeof(kTileCfgs) / sizeof(kTileCfgs[0]);

template <typename T, int PHYS, int MODE, int TX, int TY, int NT>
int launch_batched_cfg(const StageArgs<T>* args, const BatchTile* tiles, int ntiles, int ctas_per_sm, int nsm,
                       cudaStream_t s) {
    using Pol = typename PolOf<PHYS>::type;
    auto kern = stage_box_batched<T, Pol, MODE, TX, TY, NT>;
    int occ = 0;
    PHIX_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, NT, 0));
    int per_sm = ctas_per_sm > 0 ? std::min(ctas_per_sm, std::max(occ, 1)) : std::max(occ, 1);
    int grid = std::min(ntiles, nsm * per_sm);
    if (grid < 1) grid = 1;
    kern<<<grid, NT, 0, s>>>(args, tiles, ntiles, Pol{});
    PHIX_LAUNCH_CHECK("stage_box_batched");
    return PHIX_OK;
}

// One launch per RK4 step over the whole batch (step2d.cuh): 128x32 tiles,
// 512 threads, one CTA per tile of the step tile list.
constexpr int BST_TX = 128, BST_TY = 32, BST_NT = 512;

template <typename T, int PHYS>
int batched_step_cfg(bool prepare, const StepArgs<T>* args, const BatchTile* tiles, int ntiles, int nsm,
                     cudaStream_t s) {
    using Pol = typename PolOf<PHYS>::type;
    using G = Step2D<T, Pol, BST_TX, BST_TY>;
    auto kern = step_box_batched<T, Pol, BST_TX, BST_TY, BST_NT>;
    if (G::smem_bytes() > 227 * 1024) {
        if (prepare) return PHIX_OK;
        set_error("batch: the one-launch step tile does not fit in shared memory");
        return PHIX_ERR_UNSUPPORTED;
    }
    if (prepare) {
        PHIX_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::smem_bytes()));
        return PHIX_OK;
    }
    (void)nsm;
    if (ntiles < 1) return PHIX_OK;
    kern<<<ntiles, BST_NT, G::smem_bytes(), s>>>(args, tiles, Pol{});
    PHIX_LAUNCH_CHECK("step_box_batched");
    return PHIX_OK;
}

template <typename T>
int batched_step(int phys, bool prepare, const StepArgs<T>* args, const BatchTile* tiles, int ntiles, int nsm,
                 cudaStream_t s) {
    if (phys == PHIX_PHYS_AC) return batched_step_cfg<T, PHIX_PHYS_AC>(prepare, args, tiles, ntiles, nsm, s);
    return batched_step_cfg<T, PHIX_PHYS_CH>(prepare, args, tiles, ntiles, nsm, s);
}

// The pair kernels (step2d_pair.cuh) where every instance is CH with four
// periodic sides: tiles of 128x32 (FP32) or 64x32 (FP64), 8 row blocks; 32
// rows divide every grid size of the batched CH workload.
template <typename T> struct BatchPair;
template <> struct BatchPair<float> { static constexpr int TX = 128, TY = 32, NRP = 8; };
template <> struct BatchPair<double> { static constexpr int TX = 64, TY = 32, NRP = 8; };

template <typename T, int NS>
int batched_pair_ns(bool prepare, const StepArgs<T>* args, const BatchTile* tiles, int ntiles, cudaStream_t s) {
    using C = BatchPair<T>;
    using G = StepPair<T, C::TX, C::TY, C::NRP, NS>;
    static_assert(G::smem_bytes() <= 227 * 1024, "batched pair tile exceeds shared memory");
    auto kern = step_pair_batched<T, C::TX, C::TY, C::NRP, NS>;
    if (prepare) {
        PHIX_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::smem_bytes()));
        return PHIX_OK;
    }
    if (ntiles < 1) return PHIX_OK;
    kern<<<ntiles, G::NT, G::smem_bytes(), s>>>(args, tiles);
    PHIX_LAUNCH_CHECK("step_pair_batched");
    return PHIX_OK;
}

// depth: time steps per launch (2: the temporally blocked pair kernel)
template <typename T>
int batched_pair(bool prepare, const StepArgs<T>* args, const BatchTile* tiles, int ntiles, cudaStream_t s,
                 int depth = 1) {
    if (prepare) {
        int rc = batched_pair_ns<T, 1>(true, args, tiles, ntiles, s);
        return rc ? rc : batched_pair_ns<T, 2>(true, args, tiles, ntiles, s);
    }
    return depth == 2 ? batched_pair_ns<T, 2>(false, args, tiles, ntiles, s)
                      : batched_pair_ns<T, 1>(false, args, tiles, ntiles, s);
}

template <typename T, int PHYS, int MODE>
int launch_batched_mode(int cfg, const StageArgs<T>* args, const BatchTile* tiles, int ntiles, int cps, int nsm,
                        cudaStream_t s) {
    switch (cfg) {
        case 0: return launch_batched_cfg<T, PHYS, MODE, 64, 16, 256>(args, tiles, ntiles, cps, nsm, s);
        case 1: return launch_batched_cfg<T, PHYS, MODE, 32, 16, 256>(args, tiles, ntiles, cps, nsm, s);
        case 2: return launch_batched_cfg<T, PHYS, MODE, 128, 8, 256>(args, tiles, ntiles, cps, nsm, s);
        case 3: return launch_batched_cfg<T, PHYS, MODE, 64, 8, 256>(args, tiles, ntiles, cps, nsm, s);
        case 4: return launch_batched_cfg<T, PHYS, MODE, 32, 32, 256>(args, tiles, ntiles, cps, nsm, s);
        case 5: return launch_batched_cfg<T, PHYS, MODE, 128, 16, 256>(args, tiles, ntiles, cps, nsm, s);
    }
    set_error("batch: bad tile config %d", cfg);
    return PHIX_ERR_ARG;
}

template <typename T, int PHYS>
int launch_batched_phys(int mode, int cfg, const StageArgs<T>* args, const BatchTile* tiles, int ntiles, int cps,
                        int nsm, cudaStream_t s) {
    switch (mode) {
        case MODE_K: return launch_batched_mode<T, PHYS, MODE_K>(cfg, args, tiles, ntiles, cps, nsm, s);
        case MODE_RK4_FINAL: return launch_batched_mode<T, PHYS, MODE_RK4_FINAL>(cfg, args, tiles, ntiles, cps, nsm, s);
        default: return launch_batched_mode<T, PHYS, MODE_EULER_FINAL>(cfg, args, tiles, ntiles, cps, nsm, s);
    }
}

template <typename T>
int launch_batched(int phys, int mode, int cfg, const StageArgs<T>* args, const BatchTile* tiles, int ntiles, int cps,
                   int nsm, cudaStream_t s) {
    switch (phys) {
        case PHIX_PHYS_AC: return launch_batched_phys<T, PHIX_PHYS_AC>(mode, cfg, args, tiles, ntiles, cps, nsm, s);
        case PHIX_PHYS_CH: return launch_batched_phys<T, PHIX_PHYS_CH>(mode, cfg, args, tiles, ntiles, cps, nsm, s);
    }
    set_error("batch: physics %d not supported", phys);
    return PHIX_ERR_UNSUPPORTED;
}

// Per-tile FP64 sums of field 0 over physical cells; then per-instance sums of
// the tile partials in list order (deterministic).
template <typename T>
__global__ void __launch_bounds__(256) batch_tile_mass(const StageArgs<T>* __restrict__ args,
                                                       const BatchTile* __restrict__ tiles, int ntiles, int tx, int ty,
                                                       double* __restrict__ part) {
    __shared__ double sh[8];
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const BatchTile bt = tiles[t];
        const StageArgs<T>& A = args[bt.inst];
        double s = 0.0;
        for (int i = threadIdx.x; i < tx * ty; i += 256) {
            const int px = bt.x0 + i % tx, py = bt.y0 + i / tx;
            if (px < A.L.n[0] && py < A.L.n[1]) s += (double)A.u[0][A.L.origin + px + A.L.s[1] * py];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double v = 0.0;
            for (int w = 0; w < 8; ++w) v += sh[w];
            part[t] = v;
        }
        __syncthreads();
    }
}

// se[i] = first tile of instance i, se[ninst + 1 + i] = one past its last.
__global__ void batch_inst_sum(const double* __restrict__ part, const int* __restrict__ se, int ninst,
                               const double* __restrict__ dv, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ninst) return;
    double s = 0.0;
    for (int t = se[i]; t < se[ninst + 1 + i]; ++t) s += part[t];
    out[i] = s * dv[i];
}

}  // namespace
}  // namespace phix

using namespace phix;

struct phix_batch {
    int phys = 0, scheme = 0, prec = 0, ninst = 0, nf = 1;
    double dt = 0.0;
    size_t esz = 8;
    std::vector<phix_grid_t> grids;
    std::vector<Layout> layouts;
    std::vector<size_t> stored;
    std::vector<double> prm;          // ninst x 8
    void* pool = nullptr;             // all buffers
    std::vector<void*> st[2], kb[3];  // per instance (field 0 only: batch supports 1-field physics)
    std::vector<void*> lo[2];         // FP32: low parts of the compensated state
    int cur = 0;
    int cfg = 0, ctas_per_sm = 0, nsm = 148;
    // device-side argument tables: [stage kind][parity] -> ninst StageArgs
    void* args_dev = nullptr;
    size_t args_bytes = 0;
    BatchTile* tiles_dev = nullptr;
    int ntiles = 0, tiles_cfg = -1;
    int* first_dev = nullptr;         // instance -> first tile index (ninst+1)
    double* dv_dev = nullptr;
    double* part_dev = nullptr;
    double* mass_dev = nullptr;
    cudaStream_t cap = nullptr;
    int graph_steps = 0;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    // one launch per RK4 step (possible where every side is periodic or zero-flux)
    bool can_fuse = false, fuse_steps = false;
    bool step_pair = false;  // the fused step runs the pair kernels
    int depth = 1;           // time steps per pair-kernel launch (temporal blocking: 2)
    int graph_launches[2] = {0, 0};
    bool graph_flip[2] = {false, false};
    void* step_args_dev = nullptr;  // [parity][ninst] StepArgs
    BatchTile* step_tiles_dev = nullptr;
    int step_ntiles = 0;
};

namespace phix {
namespace {

void batch_drop_graphs(phix_batch* b) {
    for (auto& e : b->gexec)
        if (e) { cudaGraphExecDestroy(e); e = nullptr; }
}

// Tile list for tile config `cfg`: instances in descending size, so the
// persistent CTAs' round-robin walk over the list stays balanced.
int build_tiles(phix_batch* b, int cfg) {
    if (b->tiles_cfg == cfg) return PHIX_OK;
    const TileCfg tc = kTileCfgs[cfg];
    std::vector<int> order(b->ninst);
    for (int i = 0; i < b->ninst; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
        return (long long)b->grids[a].n[0] * b->grids[a].n[1] > (long long)b->grids[c].n[0] * b->grids[c].n[1];
    });
    std::vector<BatchTile> tiles;
    // tiles grouped per instance (for the mass sums) in the size order
    std::vector<std::vector<BatchTile>> per(b->ninst);
    for (int i = 0; i < b->ninst; ++i) {
        const phix_grid_t& g = b->grids[i];
        for (int y = 0; y < g.n[1]; y += tc.ty)
            for (int x = 0; x < g.n[0]; x += tc.tx) per[i].push_back({i, x, y, 0});
    }
    std::vector<int> pos(b->ninst);
    for (int oi = 0; oi < b->ninst; ++oi) {
        const int i = order[oi];
        pos[i] = (int)tiles.size();
        tiles.insert(tiles.end(), per[i].begin(), per[i].end());
    }
    // instance i's tiles are contiguous at [pos[i], pos[i] + per[i].size())
    if (b->first_dev) cudaFree(b->first_dev);
    if (b->tiles_dev) cudaFree(b->tiles_dev);
    if (b->part_dev) cudaFree(b->part_dev);
    b->first_dev = nullptr;
    b->tiles_dev = nullptr;
    b->part_dev = nullptr;
    // encode [start, end) per instance as two arrays packed: first[i] = start, first[ninst + 1 + i] = end
    std::vector<int> se(2 * (b->ninst + 1), 0);
    for (int i = 0; i < b->ninst; ++i) {
        se[i] = pos[i];
        se[b->ninst + 1 + i] = pos[i] + (int)per[i].size();
    }
    b->ntiles = (int)tiles.size();
    PHIX_TRY_CUDA(cudaMalloc(&b->tiles_dev, sizeof(BatchTile) * tiles.size()));
    PHIX_TRY_CUDA(cudaMemcpy(b->tiles_dev, tiles.data(), sizeof(BatchTile) * tiles.size(), cudaMemcpyHostToDevice));
    PHIX_TRY_CUDA(cudaMalloc(&b->first_dev, sizeof(int) * se.size()));
    PHIX_TRY_CUDA(cudaMemcpy(b->first_dev, se.data(), sizeof(int) * se.size(), cudaMemcpyHostToDevice));
    PHIX_TRY_CUDA(cudaMalloc(&b->part_dev, sizeof(double) * tiles.size()));
    b->tiles_cfg = cfg;
    batch_drop_graphs(b);
    return PHIX_OK;
}

template <typename T>
StageArgs<T>* args_table(phix_batch* b, int kind, int parity) {
    return reinterpret_cast<StageArgs<T>*>(b->args_dev) + ((size_t)kind * 2 + parity) * b->ninst;
}

// kinds: 0 = RK4 stage 1, 1 = stage 2, 2 = stage 3, 3 = RK4 final, 4 = Euler final
template <typename T>
int build_args(phix_batch* b) {
    const size_t n = (size_t)5 * 2 * b->ninst;
    std::vector<StageArgs<T>> h(n);
    memset(h.data(), 0, sizeof(StageArgs<T>) * n);
    for (int kind = 0; kind < 5; ++kind)
        for (int par = 0; par < 2; ++par)
            for (int i = 0; i < b->ninst; ++i) {
                StageArgs<T>& A = h[((size_t)kind * 2 + par) * b->ninst + i];
                const phix_grid_t& g = b->grids[i];
                A.L = b->layouts[i];
                for (int a = 0; a < 3; ++a) A.i2[a] = a < g.dim ? (T)(1.0 / (g.d[a] * g.d[a])) : (T)0;
                make_coeffs<T>(b->phys, &b->prm[8 * i], A.p);
                A.u[0] = (const T*)b->st[par][i];
                if (kind == 0) {
                    A.out[0] = (T*)b->kb[0][i];
                } else if (kind == 1 || kind == 2) {
                    A.kin[0] = (const T*)b->kb[kind - 1][i];
                    A.out[0] = (T*)b->kb[kind][i];
                    A.a = (T)(b->dt * 0.5);
                } else if (kind == 3) {
                    A.kin[0] = (const T*)b->kb[2][i];
                    A.k1[0] = (const T*)b->kb[0][i];
                    A.k2[0] = (const T*)b->kb[1][i];
                    A.out[0] = (T*)b->st[1 - par][i];
                    A.a = (T)b->dt;
                    A.dtf = (T)(b->dt / 6.0);
                } else {
                    A.out[0] = (T*)b->st[1 - par][i];
                    A.dtf = (T)b->dt;
                }
                if (kind >= 3 && b->lo[0][i]) {
                    A.ulo[0] = (const T*)b->lo[par][i];
                    A.outlo[0] = (T*)b->lo[1 - par][i];
                }
            }
    if (!b->args_dev) {
        b->args_bytes = sizeof(StageArgs<T>) * n;
        PHIX_TRY_CUDA(cudaMalloc(&b->args_dev, b->args_bytes));
    }
    PHIX_TRY_CUDA(cudaMemcpy(b->args_dev, h.data(), sizeof(StageArgs<T>) * n, cudaMemcpyHostToDevice));
    return PHIX_OK;
}

// StepArgs per parity and instance, and the tile list of the step kernel.
template <typename T>
int build_step(phix_batch* b) {
    std::vector<StepArgs<T>> h((size_t)2 * b->ninst);
    memset(h.data(), 0, sizeof(StepArgs<T>) * h.size());
    for (int par = 0; par < 2; ++par)
        for (int i = 0; i < b->ninst; ++i) {
            StepArgs<T>& B = h[(size_t)par * b->ninst + i];
            const phix_grid_t& g = b->grids[i];
            B.S.L = b->layouts[i];
            for (int a = 0; a < 3; ++a) B.S.i2[a] = a < g.dim ? (T)(1.0 / (g.d[a] * g.d[a])) : (T)0;
            make_coeffs<T>(b->phys, &b->prm[8 * i], B.S.p);
            B.S.u[0] = (const T*)b->st[par][i];
            B.S.out[0] = (T*)b->st[1 - par][i];
            B.S.dtf = (T)(b->dt / 6.0);
            if (b->lo[0][i]) {
                B.S.ulo[0] = (const T*)b->lo[par][i];
                B.S.outlo[0] = (T*)b->lo[1 - par][i];
            }
            B.dt2 = (T)(b->dt * 0.5);
            B.dt = (T)b->dt;
        }
    PHIX_TRY_CUDA(cudaMalloc(&b->step_args_dev, sizeof(StepArgs<T>) * h.size()));
    PHIX_TRY_CUDA(cudaMemcpy(b->step_args_dev, h.data(), sizeof(StepArgs<T>) * h.size(), cudaMemcpyHostToDevice));
    // tiles, largest instances first (the persistent walk stays balanced)
    std::vector<int> order(b->ninst);
    for (int i = 0; i < b->ninst; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
        return (long long)b->grids[a].n[0] * b->grids[a].n[1] > (long long)b->grids[c].n[0] * b->grids[c].n[1];
    });
    b->step_pair = b->phys == PHIX_PHYS_CH;
    for (int i = 0; i < b->ninst && b->step_pair; ++i) b->step_pair = step_pair_supported(b->layouts[i], 2);
    const int tx = b->step_pair ? BatchPair<T>::TX : BST_TX, ty = b->step_pair ? BatchPair<T>::TY : BST_TY;
    std::vector<BatchTile> tiles;
    for (int i : order)
        for (int y = 0; y < b->grids[i].n[1]; y += ty)
            for (int x = 0; x < b->grids[i].n[0]; x += tx) tiles.push_back({i, x, y, 0});
    b->step_ntiles = (int)tiles.size();
    PHIX_TRY_CUDA(cudaMalloc(&b->step_tiles_dev, sizeof(BatchTile) * tiles.size()));
    PHIX_TRY_CUDA(cudaMemcpy(b->step_tiles_dev, tiles.data(), sizeof(BatchTile) * tiles.size(), cudaMemcpyHostToDevice));
    if (b->step_pair) return batched_pair<T>(true, nullptr, nullptr, 0, nullptr);
    return batched_step<T>(b->phys, true, nullptr, nullptr, 0, 0, nullptr);
}

template <typename T>
int batch_step(phix_batch* b, cudaStream_t s, int depth) {
    const int par = b->cur;
    int rc;
    if (b->fuse_steps) {
        const StepArgs<T>* args = reinterpret_cast<const StepArgs<T>*>(b->step_args_dev) + (size_t)par * b->ninst;
        rc = b->step_pair ? batched_pair<T>(false, args, b->step_tiles_dev, b->step_ntiles, s, depth)
                          : batched_step<T>(b->phys, false, args, b->step_tiles_dev, b->step_ntiles, b->nsm, s);
        if (rc) return rc;
    } else if (b->scheme == PHIX_EULER) {
        rc = launch_batched<T>(b->phys, MODE_EULER_FINAL, b->cfg, args_table<T>(b, 4, par), b->tiles_dev, b->ntiles,
                               b->ctas_per_sm, b->nsm, s);
        if (rc) return rc;
    } else {
        for (int kind = 0; kind < 3; ++kind)
            if ((rc = launch_batched<T>(b->phys, MODE_K, b->cfg, args_table<T>(b, kind, par), b->tiles_dev, b->ntiles,
                                        b->ctas_per_sm, b->nsm, s)))
                return rc;
        if ((rc = launch_batched<T>(b->phys, MODE_RK4_FINAL, b->cfg, args_table<T>(b, 3, par), b->tiles_dev,
                                    b->ntiles, b->ctas_per_sm, b->nsm, s)))
            return rc;
    }
    b->cur = 1 - par;
    return PHIX_OK;
}

int batch_depth(const phix_batch* b) { return b->fuse_steps && b->step_pair ? b->depth : 1; }

int batch_launches_per_step(const phix_batch* b) { return b->scheme == PHIX_RK4 && !b->fuse_steps ? 4 : 1; }

// n time steps; with depth 2, pairs of steps per launch and an odd
// remainder as one single-step launch
int batch_steps(phix_batch* b, int n, cudaStream_t s, int* launches = nullptr) {
    const int d = batch_depth(b);
    for (int i = 0; i < n;) {
        const int k = d == 2 && n - i >= 2 ? 2 : 1;
        int rc = b->prec == PHIX_F32 ? batch_step<float>(b, s, k) : batch_step<double>(b, s, k);
        if (rc) return rc;
        if (launches) *launches += batch_launches_per_step(b);
        i += k;
    }
    return PHIX_OK;
}

int batch_replay(phix_batch* b, cudaStream_t s) {
    const int parity = b->cur;
    if (!b->gexec[parity]) {
        cudaGraph_t graph = nullptr;
        PHIX_TRY_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
        int rc, launches = 0;
        {
            LaunchCountPause pause;  // recorded, not launched: the replay below counts them
            rc = batch_steps(b, b->graph_steps, b->cap, &launches);
        }
        cudaError_t e = cudaStreamEndCapture(b->cap, &graph);
        b->graph_flip[parity] = b->cur != parity;  // each launch swaps the state buffers
        b->graph_launches[parity] = launches;
        b->cur = parity;
        if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
        if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&b->gexec[parity], graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return cuda_status(e, "cudaGraphInstantiate");
    }
    PHIX_TRY_CUDA(cudaGraphLaunch(b->gexec[parity], s));
    count_launch(b->graph_launches[parity]);
    if (b->graph_flip[parity]) b->cur = 1 - parity;
    return PHIX_OK;
}

}  // namespace
}  // namespace phix

extern "C" {

int phix_batch_create(phix_batch_t** out, int phys, int scheme, int precision, int ninst, const phix_grid_t* grids,
                      const double* prm, double dt) {
    if (!out || !grids || !prm || ninst < 1) { set_error("batch_create: bad argument"); return PHIX_ERR_ARG; }
    *out = nullptr;
    if (phys != PHIX_PHYS_AC && phys != PHIX_PHYS_CH) {
        set_error("batch: single-field physics only (AC, CH)");
        return PHIX_ERR_UNSUPPORTED;
    }
    if (scheme != PHIX_EULER && scheme != PHIX_RK4) { set_error("batch: unknown scheme %d", scheme); return PHIX_ERR_ARG; }
    if (precision != PHIX_F32 && precision != PHIX_F64) { set_error("batch: unknown precision"); return PHIX_ERR_ARG; }
    auto* b = new (std::nothrow) phix_batch();
    if (!b) { set_error("out of host memory"); return PHIX_ERR_ARG; }
    b->phys = phys;
    b->scheme = scheme;
    b->prec = precision;
    b->ninst = ninst;
    b->dt = dt;
    b->esz = precision == PHIX_F32 ? 4 : 8;
    b->grids.assign(grids, grids + ninst);
    b->layouts.resize(ninst);
    b->stored.resize(ninst);
    b->prm.assign(prm, prm + 8 * (size_t)ninst);
    for (int i = 0; i < ninst; ++i) {
        int rc = validate_grid(&grids[i], &b->layouts[i], &b->stored[i]);
        if (!rc && grids[i].dim != 2) { set_error("batch: instance %d is not 2-D", i); rc = PHIX_ERR_UNSUPPORTED; }
        if (rc) { delete b; return rc; }
    }
    // pool: per instance 2 states (+ 2 low parts in FP32) + 3 k (RK4), each
    // padded to 256 bytes
    const int nlo = precision == PHIX_F32 ? 2 : 0;
    const int nbuf = (scheme == PHIX_RK4 ? 5 : 2) + nlo;
    size_t total = 0;
    std::vector<size_t> off(ninst);
    for (int i = 0; i < ninst; ++i) {
        off[i] = total;
        total += nbuf * ((b->stored[i] * b->esz + 255) / 256 * 256);
    }
    cudaError_t e = cudaMalloc(&b->pool, total);
    if (e != cudaSuccess) { delete b; return cuda_status(e, "cudaMalloc(batch pool)"); }
    cudaMemset(b->pool, 0, total);
    for (int k = 0; k < 2; ++k) b->st[k].resize(ninst);
    for (int k = 0; k < 2; ++k) b->lo[k].resize(ninst, nullptr);
    for (int k = 0; k < 3; ++k) b->kb[k].resize(ninst, nullptr);
    for (int i = 0; i < ninst; ++i) {
        const size_t sz = (b->stored[i] * b->esz + 255) / 256 * 256;
        char* base = (char*)b->pool + off[i];
        b->st[0][i] = base;
        b->st[1][i] = base + sz;
        if (scheme == PHIX_RK4)
            for (int k = 0; k < 3; ++k) b->kb[k][i] = base + (2 + k) * sz;
        if (nlo) {
            char* lb = base + (nbuf - 2) * sz;
            b->lo[0][i] = lb;
            b->lo[1][i] = lb + sz;
        }
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, dev);
    int rc = b->prec == PHIX_F32 ? build_args<float>(b) : build_args<double>(b);
    if (!rc) rc = build_tiles(b, 0);
    // one launch per RK4 step: available, and the default, for batches whose
    // sides are all periodic or zero-flux (phix_batch_set_fusion)
    bool steppable = scheme == PHIX_RK4;
    for (int i = 0; i < ninst && steppable; ++i) steppable = step2d_supported(b->layouts[i], grids[i].dim);
    if (!rc && steppable) {
        rc = b->prec == PHIX_F32 ? build_step<float>(b) : build_step<double>(b);
        b->can_fuse = b->fuse_steps = rc == PHIX_OK;
    }
    if (!rc) {
        std::vector<double> dv(ninst, 1.0);
        for (int i = 0; i < ninst; ++i)
            for (int a = 0; a < grids[i].dim; ++a) dv[i] *= grids[i].d[a];
        e = cudaMalloc(&b->dv_dev, sizeof(double) * ninst);
        if (e == cudaSuccess) e = cudaMemcpy(b->dv_dev, dv.data(), sizeof(double) * ninst, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMalloc(&b->mass_dev, sizeof(double) * ninst);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
        if (e != cudaSuccess) rc = cuda_status(e, "batch_create");
    }
    if (rc) { phix_batch_destroy(b); return rc; }
    *out = b;
    return PHIX_OK;
}

int phix_batch_launches_per_step(const phix_batch_t* b) {
    if (!b) return -1;
    return b->scheme == PHIX_RK4 && !b->fuse_steps ? 4 : 1;
}

int phix_batch_destroy(phix_batch_t* b) {
    if (!b) return PHIX_OK;
    batch_drop_graphs(b);
    if (b->pool) cudaFree(b->pool);
    if (b->args_dev) cudaFree(b->args_dev);
    if (b->tiles_dev) cudaFree(b->tiles_dev);
    if (b->first_dev) cudaFree(b->first_dev);
    if (b->part_dev) cudaFree(b->part_dev);
    if (b->dv_dev) cudaFree(b->dv_dev);
    if (b->mass_dev) cudaFree(b->mass_dev);
    if (b->step_args_dev) cudaFree(b->step_args_dev);
    if (b->step_tiles_dev) cudaFree(b->step_tiles_dev);
    if (b->cap) cudaStreamDestroy(b->cap);
    delete b;
    return PHIX_OK;
}

int phix_batch_load(phix_batch_t* b, int inst, const double* field, int from_host, void* stream) {
    if (!b || !field || inst < 0 || inst >= b->ninst) { set_error("batch_load: bad argument"); return PHIX_ERR_ARG; }
    cudaStream_t s = (cudaStream_t)stream;
    const size_t S = b->stored[inst];
    for (int k = 0; k < 2; ++k) {
        void* dst = b->st[k][inst];
        if (b->prec == PHIX_F64) {
            PHIX_TRY_CUDA(cudaMemcpyAsync(dst, field, S * 8, from_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
        } else {
            if (from_host) {
                std::vector<float> th(S), tl(S);
                for (size_t q = 0; q < S; ++q) {
                    th[q] = (float)field[q];
                    tl[q] = (float)(field[q] - (double)th[q]);
                }
                PHIX_TRY_CUDA(cudaMemcpyAsync(dst, th.data(), S * 4, cudaMemcpyHostToDevice, s));
                PHIX_TRY_CUDA(cudaMemcpyAsync(b->lo[k][inst], tl.data(), S * 4, cudaMemcpyHostToDevice, s));
                PHIX_TRY_CUDA(cudaStreamSynchronize(s));
            } else {
                int rc = convert_f64_split((float*)dst, (float*)b->lo[k][inst], field, S, s);
                if (rc) return rc;
            }
        }
    }
    return PHIX_OK;
}

int phix_batch_store(phix_batch_t* b, int inst, double* field, int to_host, void* stream) {
    if (!b || !field || inst < 0 || inst >= b->ninst) { set_error("batch_store: bad argument"); return PHIX_ERR_ARG; }
    cudaStream_t s = (cudaStream_t)stream;
    const size_t S = b->stored[inst];
    const void* src = b->st[b->cur][inst];
    if (b->prec == PHIX_F64) {
        PHIX_TRY_CUDA(cudaMemcpyAsync(field, src, S * 8, to_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s));
        if (to_host) PHIX_TRY_CUDA(cudaStreamSynchronize(s));
        return PHIX_OK;
    }
    const void* lsrc = b->lo[b->cur][inst];
    if (to_host) {
        std::vector<float> th(S), tl(S);
        PHIX_TRY_CUDA(cudaMemcpyAsync(th.data(), src, S * 4, cudaMemcpyDeviceToHost, s));
        PHIX_TRY_CUDA(cudaMemcpyAsync(tl.data(), lsrc, S * 4, cudaMemcpyDeviceToHost, s));
        PHIX_TRY_CUDA(cudaStreamSynchronize(s));
        for (size_t q = 0; q < S; ++q) field[q] = (double)th[q] + (double)tl[q];
        return PHIX_OK;
    }
    return convert_pair_to_f64(field, (const float*)src, (const float*)lsrc, S, s);
}

int phix_batch_set_tiles(phix_batch_t* b, int tile_cfg, int ctas_per_sm) {
    if (!b || tile_cfg < 0 || tile_cfg >= kNumTileCfgs || ctas_per_sm < 0) {
        set_error("batch_set_tiles: bad argument");
        return PHIX_ERR_ARG;
    }
    int rc = build_tiles(b, tile_cfg);
    if (rc) return rc;
    b->cfg = tile_cfg;
    b->ctas_per_sm = ctas_per_sm;
    batch_drop_graphs(b);
    return PHIX_OK;
}

int phix_batch_get_tiles(const phix_batch_t* b, int* tile_cfg, int* ctas_per_sm, int* ntiles) {
    if (!b) { set_error("batch_get_tiles: NULL"); return PHIX_ERR_ARG; }
    if (tile_cfg) *tile_cfg = b->cfg;
    if (ctas_per_sm) *ctas_per_sm = b->ctas_per_sm;
    if (ntiles) *ntiles = b->ntiles;
    return PHIX_OK;
}

int phix_batch_set_fusion(phix_batch_t* b, int one_launch_per_step) {
    if (!b) { set_error("batch_set_fusion: NULL batch"); return PHIX_ERR_ARG; }
    const bool f = one_launch_per_step != 0;
    if (f && !b->can_fuse) {
        set_error("batch_set_fusion: one launch per step needs RK4 and periodic or zero-flux sides everywhere");
        return PHIX_ERR_UNSUPPORTED;
    }
    if (f != b->fuse_steps) {
        batch_drop_graphs(b);
        b->fuse_steps = f;
    }
    return PHIX_OK;
}

int phix_batch_set_depth(phix_batch_t* b, int depth) {
    if (!b || (depth != 1 && depth != 2)) { set_error("batch_set_depth: bad batch or depth (1 or 2)"); return PHIX_ERR_ARG; }
    if (depth == 2 && !b->step_pair) {
        set_error("batch_set_depth: two steps per launch need the pair kernels (CH, four periodic sides)");
        return PHIX_ERR_UNSUPPORTED;
    }
    if (depth != b->depth) {
        batch_drop_graphs(b);
        b->depth = depth;
    }
    return PHIX_OK;
}

int phix_batch_depth(const phix_batch_t* b) { return b ? batch_depth(b) : -1; }

int phix_batch_set_graph(phix_batch_t* b, int steps_per_graph) {
    if (!b || steps_per_graph < 0) { set_error("batch_set_graph: bad argument"); return PHIX_ERR_ARG; }
    batch_drop_graphs(b);
    b->graph_steps = steps_per_graph;
    return PHIX_OK;
}

int phix_batch_advance(phix_batch_t* b, int nsteps, void* stream) {
    if (!b || nsteps < 0) { set_error("batch_advance: bad argument"); return PHIX_ERR_ARG; }
    cudaStream_t s = (cudaStream_t)stream;
    int rc;
    if (b->graph_steps > 0)
        while (nsteps >= b->graph_steps) {
            if ((rc = batch_replay(b, s))) return rc;
            nsteps -= b->graph_steps;
        }
    return batch_steps(b, nsteps, s);
}

int phix_batch_autotune(phix_batch_t* b, int trial_steps, double* best_ms) {
    if (!b || trial_steps < 1) { set_error("batch_autotune: bad argument"); return PHIX_ERR_ARG; }
    // The state evolves during trials; save and restore it so tuning is invisible.
    const int cur0 = b->cur;
    const int parts = b->lo[0][0] ? 2 : 1;
    size_t bytes = 0;
    for (int i = 0; i < b->ninst; ++i) bytes += parts * b->stored[i] * b->esz;
    void* save = nullptr;
    PHIX_TRY_CUDA(cudaMalloc(&save, bytes));
    size_t o = 0;
    for (int i = 0; i < b->ninst; ++i)
        for (int q = 0; q < parts; ++q) {
            const void* src = q ? b->lo[cur0][i] : b->st[cur0][i];
            PHIX_TRY_CUDA(cudaMemcpy((char*)save + o, src, b->stored[i] * b->esz, cudaMemcpyDeviceToDevice));
            o += b->stored[i] * b->esz;
        }
    const int old_graph = b->graph_steps;
    b->graph_steps = 0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    int best_cfg = 0, best_cps = 0;
    bool best_fused = false;
    const int cps_options[] = {0, 2, 4};
    int rc = PHIX_OK;
    auto trial = [&](float* ms) {
        int r = batch_steps(b, batch_depth(b), 0);  // warm-up
        if (r) return r;
        cudaEventRecord(e0, 0);
        if ((r = batch_steps(b, trial_steps, 0))) return r;
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(ms, e0, e1);
        return PHIX_OK;
    };
    // one launch per stage: every tile shape x CTA count
    b->fuse_steps = false;
    for (int cfg = 0; cfg < kNumTileCfgs && !rc; ++cfg) {
        for (int cps : cps_options) {
            float ms = 0.f;
            if ((rc = phix_batch_set_tiles(b, cfg, cps)) || (rc = trial(&ms))) break;
            if (ms < best) { best = ms; best_cfg = cfg; best_cps = cps; }
        }
    }
    // one launch per RK4 step, and (pair kernels) two steps per launch
    int best_depth = b->depth;
    if (!rc && b->can_fuse) {
        const int depth0 = b->depth;
        for (int d = 1; d <= (b->step_pair ? 2 : 1) && !rc; ++d) {
            float ms = 0.f;
            b->fuse_steps = true;
            b->depth = d;
            rc = trial(&ms);
            b->fuse_steps = false;
            if (!rc && ms < best) { best = ms; best_fused = true; best_depth = d; }
        }
        b->depth = depth0;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // restore the state into the buffer that was current
    b->cur = cur0;
    o = 0;
    for (int i = 0; i < b->ninst; ++i)
        for (int q = 0; q < parts; ++q) {
            void* dst = q ? b->lo[cur0][i] : b->st[cur0][i];
            cudaMemcpy(dst, (char*)save + o, b->stored[i] * b->esz, cudaMemcpyDeviceToDevice);
            o += b->stored[i] * b->esz;
        }
    cudaFree(save);
    b->graph_steps = old_graph;
    if (rc) return rc;
    rc = phix_batch_set_tiles(b, best_cfg, best_cps);
    if (!rc) rc = phix_batch_set_fusion(b, best_fused ? 1 : 0);
    if (!rc && best_fused) rc = phix_batch_set_depth(b, best_depth);
    if (best_ms) *best_ms = best / trial_steps;
    return rc;
}

int phix_batch_mass(phix_batch_t* b, double* masses) {
    if (!b || !masses) { set_error("batch_mass: NULL"); return PHIX_ERR_ARG; }
    const TileCfg tc = kTileCfgs[b->tiles_cfg];
    const int grid = std::min(b->ntiles, b->nsm * 8);
    if (b->prec == PHIX_F32)
        batch_tile_mass<float><<<grid, 256>>>(args_table<float>(b, 0, b->cur), b->tiles_dev, b->ntiles, tc.tx, tc.ty,
                                              b->part_dev);
    else
        batch_tile_mass<double><<<grid, 256>>>(args_table<double>(b, 0, b->cur), b->tiles_dev, b->ntiles, tc.tx,
                                               tc.ty, b->part_dev);
    PHIX_LAUNCH_CHECK("batch_tile_mass");
    batch_inst_sum<<<(b->ninst + 127) / 128, 128>>>(b->part_dev, b->first_dev, b->ninst, b->dv_dev, b->mass_dev);
    PHIX_LAUNCH_CHECK("batch_inst_sum");
    PHIX_TRY_CUDA(cudaMemcpy(masses, b->mass_dev, sizeof(double) * b->ninst, cudaMemcpyDeviceToHost));
    return PHIX_OK;
}

}  // extern "C"
