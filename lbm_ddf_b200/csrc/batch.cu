// batch.cu — many Rayleigh–Bénard cases advanced together.
//
// A batch is a set of cases (any grids, Ra, Pr, collision models; one
// storage format; periodic sides) on one device.  The members are grouped by
// AA layout and collision model; one launch of batch_step_kernel per
// non-empty group (normally one: members move through the layouts in step)
// advances the group's members by one step.  Their nodes are cut into tiles
// of kTileRounds x BLOCK nodes, numbered case after case; blocks walk the tile list with a
// grid stride (persistent blocks, BLOCKS_PER_SM x 148 of them, or one block
// per tile), find each tile's case by a binary search over the tiles' prefix
// sums held in shared memory, and apply the same node update as the
// single-case kernel (step.cuh update_node) with that case's parameters.  A
// kernel instance holds the code of one layout and one model only, so it
// needs no more registers than the single-case kernel.  A case's result
// does not depend on the other members.
//
// Repeated steps are captured once into a CUDA graph (the launches of every
// step, alternating layouts) and replayed.  The launch shape (block size and
// grid) is chosen by lbm_batch_autotune, which times each candidate on real
// steps of the batch: every shape computes the same per-node arithmetic, so
// no step is wasted.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <new>
#include <vector>

#include "internal.h"
#include "step.cuh"

using namespace lbm;
using namespace lbm_internal;

namespace lbm {

constexpr int kMaxBatch = 2048;    // members per batch (tile prefix sums in shared memory)
constexpr int kLanes = 8;          // streams of the one-kernel-per-member launch
// A tile is kTileRounds rounds of BLOCK nodes of one member, so the member
// lookup (binary search, descriptor) is paid once per kTileRounds nodes a
// thread updates (96-case FP16S ensemble on B200: 19.3, 19.9, 20.5 and 20.6
// GLUPS at 1, 2, 4 and 8 rounds; FP32 unchanged).
constexpr int kTileRounds = 4;

// Per-member descriptor, read by every block that works on the member.
// It provides what update_node needs (the accessor interface of StepArgs).
template <class S> struct BatchCase {
    using R = typename Codec<S>::R;
    using P = typename Codec<S>::P;
    S *f, *g;            // population row 0; row k at + k*ps
    S *f_st, *g_st;      // the same arrays, for stores (see StepArgs)
    P *phip;
    uint32_t ps, nodes;
    int32_t lx, ly, lz, swapped;
    FastDiv div_lx, div_ly;
    R tau, tauc, rcp_tau, rcp_tauc, rcp_rt;
    R omega_f, omega_g, force_fac, gb, t0, t_hot, t_cold, phi_fix;
    R t_top, t_dy;       // 16-bit storage: the conduction-profile shift (step.cuh shift0)
    int32_t use_phi_fix, pad;

    // element (k * ps + j) * elem_stride of the population array, indexed
    // in 32 bits (a member has 27 ps elem_stride < 2^32 elements per
    // array): one multiply-add per access and no 64-bit row addresses held
    // in registers
    template <class I> __device__ __forceinline__ const S *ldp(int which, int k, I j) const {
        return (which ? g : f) + ((uint32_t)k * ps + (uint32_t)j) * elem_stride<S>();
    }
    template <class I> __device__ __forceinline__ S ld(int which, int k, I j) const { return *ldp(which, k, j); }
    template <class I> __device__ __forceinline__ S &st(int which, int k, I j) const {
        return (which ? g_st : f_st)[((uint32_t)k * ps + (uint32_t)j) * elem_stride<S>()];
    }
    // 16-bit storage: the (f_k, g_k) pair of node j as one 32-bit word
    template <class I, class SS = S> __device__ __forceinline__ typename Pack16<SS>::T ld2(int k, I j) const {
        return reinterpret_cast<const typename Pack16<SS>::T *>(f)[(uint32_t)k * ps + (uint32_t)j];
    }
    template <class I, class SS = S> __device__ __forceinline__ typename Pack16<SS>::T &st2(int k, I j) const {
        return reinterpret_cast<typename Pack16<SS>::T *>(f_st)[(uint32_t)k * ps + (uint32_t)j];
    }
};

// Resident threads per SM the batch kernel's registers are sized for: those
// of the single-case kernel, except 512 (128 registers) for 16-bit storage:
// one 256^3 FP16S case through the batch kernel on B200 ran at 15.7 GLUPS
// with 640 threads (96 registers) and 19.2-20.9 with 512.
template <class S> constexpr int batch_threads_per_sm() {
    return sizeof(S) == 2 ? 512 : StepOccupancy<S>::value * 128;
}
template <class S, int BLOCK> struct BatchOccupancy {
    static constexpr int value = batch_threads_per_sm<S>() / BLOCK > 0 ? batch_threads_per_sm<S>() / BLOCK : 1;
};

// Advances the members cases[0 .. ncases) of one group, all in layout
// SWAPPED and collision model COLL, by one step.  tile_start[i] is the first
// tile of member i (tile numbers are batch-wide; the group owns tiles
// [tile_start[0], tile_start[ncases])).
template <class S, int BLOCK, bool SWAPPED, int COLL>
__global__ void __launch_bounds__(BLOCK, BatchOccupancy<S, BLOCK>::value)
    batch_step_kernel(const BatchCase<S> *__restrict__ cases, int ncases, const uint32_t *__restrict__ tile_start) {
    __shared__ uint32_t s_start[kMaxBatch + 1];
    for (int i = threadIdx.x; i <= ncases; i += BLOCK) s_start[i] = tile_start[i];
    __syncthreads();
    const uint32_t end = s_start[ncases];
    for (uint32_t t = s_start[0] + blockIdx.x; t < end; t += gridDim.x) {
        int lo = 0, hi = ncases;   // the member c with s_start[c] <= t < s_start[c+1]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (s_start[mid] <= t) lo = mid;
            else hi = mid;
        }
        const BatchCase<S> &cs = cases[lo];
        const uint32_t u0 = (t - s_start[lo]) * (BLOCK * kTileRounds) + threadIdx.x;
#pragma unroll 1
        for (int r = 0; r < kTileRounds; r++) {
            const uint32_t u = u0 + r * BLOCK;
            if (u < cs.nodes) update_node<S, SWAPPED, true, COLL>(cs, u);
        }
    }
}

}  // namespace lbm

struct lbm_batch {
    int device = 0;
    int32_t storage = LBM_STORE_F32;
    std::vector<lbm_case *> members;
    int32_t block = 128;           // tile size = threads per block
    int32_t blocks_per_sm = 0;     // 0: one block per tile
    bool use_graph = true;
    // device copies of the descriptors and tile prefix sums
    void *d_cases = nullptr;
    uint32_t *d_start = nullptr;
    int capacity = 0;
    // Member groups (descriptor order): bit 0 = the member's layout differs
    // from the batch's phase, bit 1 = regularised collision.  Every step
    // flips all layouts and the phase together, so groups stay fixed.
    int group_first[4] = {0, 0, 0, 0}, group_count[4] = {0, 0, 0, 0};
    int phase = 0;
    bool dirty = true;             // descriptors need rebuilding / uploading
    std::vector<unsigned char> h_cases;
    std::vector<uint32_t> h_start;
    // page-locked staging of the descriptor uploads, two in turn: an upload
    // is a copy on the step stream that needs no wait, and a staging buffer
    // is reused only after its event says its copy is done
    unsigned char *stage[2] = {nullptr, nullptr};
    size_t stage_cap[2] = {0, 0};
    cudaEvent_t stage_ev[2] = {nullptr, nullptr};
    bool stage_used[2] = {false, false};
    int stage_next = 0;
    // lbm_batch_observables: one record per member (device)
    lbm_observables *d_obs = nullptr;
    int obs_cap = 0;
    // captured graphs, keyed by 2 x the number of steps + the phase at
    // capture; dropped when the membership or the launch shape changes
    std::map<int, cudaGraphExec_t> graphs;
    cudaStream_t capture_stream = nullptr;
    int sm_count = 148;
    // LBM_BATCH_PER_CASE: each member's own single-case kernel, the members
    // spread round-robin over kLanes streams forked from and joined to the
    // stepping stream (created on first use)
    int32_t launch = LBM_BATCH_TILES;
    cudaStream_t lanes[kLanes] = {};
    cudaEvent_t fork_ev = nullptr, join_ev[kLanes] = {};
};

namespace {

size_t case_desc_bytes(int storage) {
    switch (storage) {
    case LBM_STORE_F64: return sizeof(BatchCase<double>);
    case LBM_STORE_F32: return sizeof(BatchCase<float>);
    case LBM_STORE_F16S: return sizeof(BatchCase<__half>);
    default: return sizeof(BatchCase<__nv_bfloat16>);
    }
}

void drop_graphs(lbm_batch *b) {
    for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
}

template <class S> BatchCase<S> describe(const lbm_case *c) {
    using R = typename Codec<S>::R;
    BatchCase<S> d;
    std::memset(&d, 0, sizeof d);
    d.f = d.f_st = (S *)c->f;
    d.g = d.g_st = (S *)c->g;
    d.phip = (typename Codec<S>::P *)c->phip;
    d.ps = (uint32_t)c->ps;
    d.nodes = (uint32_t)c->nodes;
    d.lx = c->p.lx;
    d.ly = c->p.ly;
    d.lz = c->p.lz;
    d.swapped = c->swapped ? 1 : 0;
    d.div_lx = FastDiv((uint32_t)c->p.lx);
    d.div_ly = FastDiv((uint32_t)c->p.ly);
    d.tau = (R)c->d.tau;
    d.tauc = (R)c->d.tauc;
    d.rcp_tau = (R)(1.0 / c->d.tau);
    d.rcp_tauc = (R)(1.0 / c->d.tauc);
    d.rcp_rt = (R)(1.0 / (1.0 / 3.0));
    d.omega_f = (R)(1.0 / c->d.tau);
    d.omega_g = (R)(1.0 / c->d.tauc);
    d.force_fac = (R)(1.0 - 0.5 / c->d.tau);
    d.gb = (R)(c->p.gravity * c->p.beta);
    d.t0 = (R)c->d.t0;
    d.t_top = (R)(c->p.t_hot - (c->p.t_hot - c->p.t_cold) * 0.5 / c->p.ly);
    d.t_dy = (R)((c->p.t_hot - c->p.t_cold) / c->p.ly);
    d.t_hot = (R)c->p.t_hot;
    d.t_cold = (R)c->p.t_cold;
    d.phi_fix = (R)0.5;
    d.use_phi_fix = 0;
    return d;
}

template <class Fn> int with_batch_storage(const lbm_batch *b, Fn &&fn) {
    switch (b->storage) {
    case LBM_STORE_F64: return fn((double *)nullptr);
    case LBM_STORE_F32: return fn((float *)nullptr);
    case LBM_STORE_F16S: return fn((__half *)nullptr);
    case LBM_STORE_BF16S: return fn((__nv_bfloat16 *)nullptr);
    }
    return fail(LBM_ERR_ARG, "bad storage");
}

int group_of(const lbm_batch *b, const lbm_case *c) {
    return ((c->swapped ? 1 : 0) ^ b->phase) | (c->collision == LBM_COLLISION_REGULARIZED ? 2 : 0);
}

// Rebuilds and uploads the descriptors after a membership change.
int refresh(lbm_batch *b, cudaStream_t st) {
    if (!b->dirty) return LBM_OK;
    const int n = (int)b->members.size();
    const size_t db = case_desc_bytes(b->storage);
    if (n > b->capacity) {
        const int cap = std::max(n, std::max(16, 2 * b->capacity));
        void *dc = nullptr;
        uint32_t *ds = nullptr;
        CUDA_TRY(cudaMalloc(&dc, (size_t)cap * db));
        cudaError_t e = cudaMalloc(&ds, (size_t)(cap + 1) * sizeof(uint32_t));
        if (e != cudaSuccess) {
            cudaFree(dc);
            return fail(LBM_ERR_NOMEM, "batch descriptor allocation failed");
        }
        CUDA_TRY(cudaStreamSynchronize(st));
        cudaFree(b->d_cases);
        cudaFree(b->d_start);
        b->d_cases = dc;
        b->d_start = ds;
        b->capacity = cap;
        drop_graphs(b);
    }
    std::vector<const lbm_case *> order;
    order.reserve((size_t)n);
    for (int g = 0; g < 4; g++) {
        b->group_first[g] = (int)order.size();
        for (const lbm_case *c : b->members)
            if (group_of(b, c) == g) order.push_back(c);
        b->group_count[g] = (int)order.size() - b->group_first[g];
    }
    b->h_cases.assign((size_t)n * db, 0);
    b->h_start.assign((size_t)n + 1, 0);
    uint32_t tiles = 0;
    int rc = with_batch_storage(b, [&](auto tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        for (int i = 0; i < n; i++) {
            const BatchCase<S> d = describe<S>(order[(size_t)i]);
            std::memcpy(b->h_cases.data() + (size_t)i * db, &d, db);
            b->h_start[i] = tiles;
            const int64_t tile = (int64_t)b->block * kTileRounds;
            tiles += (uint32_t)((order[(size_t)i]->nodes + tile - 1) / tile);
        }
        return LBM_OK;
    });
    if (rc) return rc;
    b->h_start[n] = tiles;
    if (n > 0) {
        // through page-locked staging: the copies run in stream order behind
        // the steps already enqueued, and the host does not wait for them
        const int i = b->stage_next;
        const size_t cb = b->h_cases.size(), sb = b->h_start.size() * sizeof(uint32_t);
        const size_t off = (cb + 255) / 256 * 256;
        if (b->stage_used[i]) CUDA_TRY(cudaEventSynchronize(b->stage_ev[i]));
        if (!b->stage_ev[i]) CUDA_TRY(cudaEventCreateWithFlags(&b->stage_ev[i], cudaEventDisableTiming));
        if (b->stage_cap[i] < off + sb) {
            if (b->stage[i]) cudaFreeHost(b->stage[i]);
            b->stage[i] = nullptr;
            b->stage_cap[i] = 0;
            const size_t cap = std::max<size_t>(2 * (off + sb), 64 * 1024);
            CUDA_TRY(cudaMallocHost((void **)&b->stage[i], cap));
            b->stage_cap[i] = cap;
        }
        std::memcpy(b->stage[i], b->h_cases.data(), cb);
        std::memcpy(b->stage[i] + off, b->h_start.data(), sb);
        CUDA_TRY(cudaMemcpyAsync(b->d_cases, b->stage[i], cb, cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(b->d_start, b->stage[i] + off, sb, cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaEventRecord(b->stage_ev[i], st));
        b->stage_used[i] = true;
        b->stage_next = 1 - i;
    }
    b->dirty = false;
    return LBM_OK;
}

unsigned grid_of(const lbm_batch *b, uint32_t tiles) {
    if (b->blocks_per_sm <= 0) return tiles;
    return (unsigned)std::min<uint64_t>(tiles, (uint64_t)b->sm_count * b->blocks_per_sm);
}

template <class S, int BLOCK, bool SW>
void launch_group(const BatchCase<S> *cases, int n, const uint32_t *start, bool reg, unsigned grid, cudaStream_t st) {
    if (reg) batch_step_kernel<S, BLOCK, SW, LBM_COLLISION_REGULARIZED><<<grid, BLOCK, 0, st>>>(cases, n, start);
    else batch_step_kernel<S, BLOCK, SW, LBM_COLLISION_BGK><<<grid, BLOCK, 0, st>>>(cases, n, start);
}

// Lane of each member for the per-case launch: members by decreasing node
// count, each onto the lane with the fewest nodes so far (longest processing
// time first), so the lanes' work is balanced.  A lane runs its members'
// steps in order, and the lanes of a captured multi-step graph progress
// independently, so the slowest lane sets the time.
std::vector<int> lane_of_members(const lbm_batch *b, int lanes) {
    const size_t n = b->members.size();
    std::vector<size_t> order(n);
    for (size_t i = 0; i < n; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t x, size_t y) { return b->members[x]->nodes > b->members[y]->nodes; });
    std::vector<int64_t> load((size_t)lanes, 0);
    std::vector<int> lane(n, 0);
    for (size_t i : order) {
        const int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        lane[i] = l;
        load[(size_t)l] += b->members[i]->nodes;
    }
    return lane;
}

// LBM_BATCH_PER_CASE: `nsteps` steps of every member, each through its own
// single-case node kernel (its parameters in the constant bank, as lbm_step
// launches it), on the lanes of lane_of_members; the lanes are forked from
// and joined to `st` by events, so captured into a graph the members' steps
// are parallel branches and the kernels of different members run
// concurrently.
int enqueue_steps_per_case(lbm_batch *b, int nsteps, cudaStream_t st) {
    if (!b->fork_ev) {
        CUDA_TRY(cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming));
        for (int l = 0; l < kLanes; l++) {
            CUDA_TRY(cudaStreamCreateWithFlags(&b->lanes[l], cudaStreamNonBlocking));
            CUDA_TRY(cudaEventCreateWithFlags(&b->join_ev[l], cudaEventDisableTiming));
        }
    }
    const int nl = std::min<int>(kLanes, (int)b->members.size());
    const std::vector<int> lane = lane_of_members(b, nl);
    CUDA_TRY(cudaEventRecord(b->fork_ev, st));
    for (int l = 0; l < nl; l++) CUDA_TRY(cudaStreamWaitEvent(b->lanes[l], b->fork_ev, 0));
    for (int s = 0; s < nsteps; s++)
        for (size_t i = 0; i < b->members.size(); i++) {
            const lbm_case *c = b->members[i];
            const int rc = enqueue_case_step(c, c->swapped != ((s & 1) != 0), b->lanes[lane[i]]);
            if (rc) return rc;
        }
    for (int l = 0; l < nl; l++) {
        CUDA_TRY(cudaEventRecord(b->join_ev[l], b->lanes[l]));
        CUDA_TRY(cudaStreamWaitEvent(st, b->join_ev[l], 0));
    }
    return LBM_OK;
}

// Enqueues `nsteps` batch steps on `st`: per step one launch per non-empty
// group, in the layout its members are in at that step.
int enqueue_steps(lbm_batch *b, int nsteps, cudaStream_t st) {
    if (b->launch == LBM_BATCH_PER_CASE) return enqueue_steps_per_case(b, nsteps, st);
    return with_batch_storage(b, [&](auto tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        const BatchCase<S> *cases = (const BatchCase<S> *)b->d_cases;
        for (int s = 0; s < nsteps; s++)
            for (int g = 0; g < 4; g++) {
                const int first = b->group_first[g], n = b->group_count[g];
                if (n == 0) continue;
                const uint32_t tiles = b->h_start[first + n] - b->h_start[first];
                const unsigned grid = grid_of(b, tiles);
                if (grid == 0) continue;
                const bool sw = ((g & 1) ^ b->phase ^ (s & 1)) != 0;
                const bool reg = (g & 2) != 0;
                const BatchCase<S> *c0 = cases + first;
                const uint32_t *s0 = b->d_start + first;
                if (b->block == 256) {
                    if (sw) launch_group<S, 256, true>(c0, n, s0, reg, grid, st);
                    else launch_group<S, 256, false>(c0, n, s0, reg, grid, st);
                } else {
                    if (sw) launch_group<S, 128, true>(c0, n, s0, reg, grid, st);
                    else launch_group<S, 128, false>(c0, n, s0, reg, grid, st);
                }
            }
        return LBM_OK;
    });
}

// Every member's layout and the batch phase flip together on odd counts,
// so the groups and descriptors stay valid.
void advance_members(lbm_batch *b, int nsteps) {
    for (lbm_case *c : b->members) {
        c->step += nsteps;
        if (nsteps & 1) c->swapped = !c->swapped;
    }
    if (nsteps & 1) b->phase ^= 1;
}

}  // namespace

void lbm_internal::batch_forget(lbm_batch *b, lbm_case *c) {
    auto it = std::find(b->members.begin(), b->members.end(), c);
    if (it != b->members.end()) {
        b->members.erase(it);
        b->dirty = true;
        drop_graphs(b);
    }
    c->batch = nullptr;
}

extern "C" {

int lbm_batch_create(int device, int32_t storage, lbm_batch **out) {
    if (!out) return fail(LBM_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (store_bytes(storage) == 0) return fail(LBM_ERR_ARG, "bad storage");
    lbm_batch *b = new (std::nothrow) lbm_batch();
    if (!b) return fail(LBM_ERR_NOMEM, "host allocation failed");
    b->device = device;
    b->storage = storage;
    DeviceGuard dg(device);
    cudaError_t e = cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) {
        delete b;
        return fail(LBM_ERR_CUDA, cudaGetErrorString(e));
    }
    *out = b;
    return LBM_OK;
}

int lbm_batch_destroy(lbm_batch *b) {
    if (!b) return LBM_OK;
    for (lbm_case *m : b->members) m->batch = nullptr;
    DeviceGuard dg(b->device);
    drop_graphs(b);
    cudaFree(b->d_cases);
    cudaFree(b->d_start);
    cudaFree(b->d_obs);
    for (int l = 0; l < kLanes; l++) {
        if (b->lanes[l]) cudaStreamDestroy(b->lanes[l]);
        if (b->join_ev[l]) cudaEventDestroy(b->join_ev[l]);
    }
    if (b->fork_ev) cudaEventDestroy(b->fork_ev);
    for (int i = 0; i < 2; i++) {
        if (b->stage_ev[i]) {
            cudaEventSynchronize(b->stage_ev[i]);
            cudaEventDestroy(b->stage_ev[i]);
        }
        if (b->stage[i]) cudaFreeHost(b->stage[i]);
    }
    if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
    delete b;
    return LBM_OK;
}

int lbm_batch_add(lbm_batch *b, lbm_case *c) {
    if (!b || !c) return fail(LBM_ERR_ARG, "NULL argument");
    if (!c->initialised) return fail(LBM_ERR_STATE, "case has no state yet");
    if (c->p.device != b->device) return fail(LBM_ERR_ARG, "case is on another device");
    if (c->p.storage != b->storage) return fail(LBM_ERR_ARG, "case storage differs from the batch's");
    if (c->p.sides != LBM_SIDES_PERIODIC) return fail(LBM_ERR_ARG, "batches run periodic-side cases only");
    if (c->rest_phi) return fail(LBM_ERR_STATE, "take the first step of a rest-state case alone before batching it");
    if (c->batch) return fail(LBM_ERR_ARG, c->batch == b ? "case is already in the batch" : "case is in another batch");
    if ((uint64_t)Q * (uint64_t)c->ps * (interleaved(c) ? 2u : 1u) >= (1ull << 32))
        return fail(LBM_ERR_ARG, "case too large for a batch (its population array must have fewer than 2^32 "
                                 "elements)");
    if ((int)b->members.size() >= kMaxBatch) return fail(LBM_ERR_ARG, "batch is full");
    b->members.push_back(c);
    c->batch = b;
    b->dirty = true;
    drop_graphs(b);
    return LBM_OK;
}

int lbm_batch_remove(lbm_batch *b, lbm_case *c) {
    if (!b || !c) return fail(LBM_ERR_ARG, "NULL argument");
    auto it = std::find(b->members.begin(), b->members.end(), c);
    if (it == b->members.end()) return fail(LBM_ERR_ARG, "case is not in the batch");
    b->members.erase(it);
    c->batch = nullptr;
    b->dirty = true;
    drop_graphs(b);
    return LBM_OK;
}

int lbm_batch_size(const lbm_batch *b, int32_t *members, uint64_t *nodes) {
    if (!b) return fail(LBM_ERR_ARG, "batch is NULL");
    if (members) *members = (int32_t)b->members.size();
    if (nodes) {
        uint64_t s = 0;
        for (const lbm_case *c : b->members) s += (uint64_t)c->nodes;
        *nodes = s;
    }
    return LBM_OK;
}

int lbm_batch_set_config(lbm_batch *b, int32_t block, int32_t blocks_per_sm, int32_t use_graph) {
    if (!b) return fail(LBM_ERR_ARG, "batch is NULL");
    if (block != 128 && block != 256) return fail(LBM_ERR_ARG, "block must be 128 or 256");
    if (blocks_per_sm < 0 || blocks_per_sm > 64) return fail(LBM_ERR_ARG, "blocks_per_sm must be 0..64");
    if (block != b->block) b->dirty = true;
    b->block = block;
    b->blocks_per_sm = blocks_per_sm;
    b->use_graph = use_graph != 0;
    drop_graphs(b);
    return LBM_OK;
}

int lbm_batch_set_launch(lbm_batch *b, int32_t launch) {
    if (!b) return fail(LBM_ERR_ARG, "batch is NULL");
    if (launch != LBM_BATCH_TILES && launch != LBM_BATCH_PER_CASE) return fail(LBM_ERR_ARG, "unknown batch launch");
    if (launch != b->launch) drop_graphs(b);
    b->launch = launch;
    return LBM_OK;
}

int lbm_batch_get_launch(const lbm_batch *b, int32_t *launch) {
    if (!b || !launch) return fail(LBM_ERR_ARG, "NULL argument");
    *launch = b->launch;
    return LBM_OK;
}

int lbm_batch_get_config(const lbm_batch *b, int32_t *block, int32_t *blocks_per_sm, int32_t *use_graph) {
    if (!b) return fail(LBM_ERR_ARG, "batch is NULL");
    if (block) *block = b->block;
    if (blocks_per_sm) *blocks_per_sm = b->blocks_per_sm;
    if (use_graph) *use_graph = b->use_graph ? 1 : 0;
    return LBM_OK;
}

int lbm_batch_step(lbm_batch *b, int32_t nsteps, void *stream) {
    if (!b) return fail(LBM_ERR_ARG, "batch is NULL");
    if (nsteps < 0) return fail(LBM_ERR_ARG, "nsteps < 0");
    if (nsteps == 0 || b->members.empty()) return LBM_OK;
    DeviceGuard dg(b->device);
    cudaStream_t st = (cudaStream_t)stream;
    int rc = refresh(b, st);
    if (rc) return rc;
    if (b->use_graph && nsteps > 1) {
        const int key = 2 * nsteps + b->phase;
        auto it = b->graphs.find(key);
        if (it == b->graphs.end()) {
            cudaGraph_t g = nullptr;
            CUDA_TRY(cudaStreamBeginCapture(b->capture_stream, cudaStreamCaptureModeThreadLocal));
            rc = enqueue_steps(b, nsteps, b->capture_stream);
            cudaError_t e = cudaStreamEndCapture(b->capture_stream, &g);
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            if (e != cudaSuccess) return fail(LBM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
            cudaGraphExec_t x = nullptr;
            e = cudaGraphInstantiate(&x, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return fail(LBM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
            it = b->graphs.emplace(key, x).first;
        }
        CUDA_TRY(cudaGraphLaunch(it->second, st));
    } else {
        rc = enqueue_steps(b, nsteps, st);
        if (rc) return rc;
        CUDA_TRY(cudaGetLastError());
    }
    advance_members(b, nsteps);
    return LBM_OK;
}

int lbm_batch_observables(lbm_batch *b, lbm_observables *out, void *stream) {
    if (!b) return fail(LBM_ERR_ARG, "batch is NULL");
    const int n = (int)b->members.size();
    if (n == 0) return LBM_OK;
    if (!out) return fail(LBM_ERR_ARG, "out is NULL");
    DeviceGuard dg(b->device);
    cudaStream_t st = (cudaStream_t)stream;
    if (n > b->obs_cap) {
        const int cap = std::max(n, std::max(16, 2 * b->obs_cap));
        lbm_observables *d = nullptr;
        CUDA_TRY(cudaMalloc(&d, (size_t)cap * sizeof(lbm_observables)));
        if (b->d_obs) {   // earlier calls may still write the old array
            cudaError_t e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) {
                cudaFree(d);
                return fail(LBM_ERR_CUDA, cudaGetErrorString(e));
            }
            cudaFree(b->d_obs);
        }
        b->d_obs = d;
        b->obs_cap = cap;
    }
    for (int i = 0; i < n; i++) {
        const lbm_case *c = b->members[(size_t)i];
        if (!c->initialised) return fail(LBM_ERR_STATE, "a member has no state");
        const int rc = enqueue_observables(c, b->d_obs + i, st);
        if (rc) return rc;
    }
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(out, b->d_obs, (size_t)n * sizeof(lbm_observables), cudaMemcpyDefault, st));
    return LBM_OK;
}

int lbm_batch_autotune(lbm_batch *b, int32_t steps_per_trial, void *stream, int32_t *block, int32_t *blocks_per_sm,
                       double *best_ms_per_step) {
    if (!b) return fail(LBM_ERR_ARG, "batch is NULL");
    if (steps_per_trial < 2 || (steps_per_trial & 1)) return fail(LBM_ERR_ARG, "steps_per_trial must be even, >= 2");
    if (b->members.empty()) return fail(LBM_ERR_STATE, "batch is empty");
    DeviceGuard dg(b->device);
    cudaStream_t st = (cudaStream_t)stream;
    // candidates: the tile walk at 2 block sizes x 5 grids, and one kernel per member
    struct Shape {
        int32_t launch, block, per_sm;
    };
    std::vector<Shape> shapes;
    for (int blk : {128, 256})
        for (int ps : {0, 4, 8, 16, 32}) shapes.push_back({LBM_BATCH_TILES, blk, ps});
    shapes.push_back({LBM_BATCH_PER_CASE, 128, 0});   // the tile shape is then unused
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    double best = 1e30;
    Shape keep{b->launch, b->block, b->blocks_per_sm};
    const bool graph = b->use_graph;
    int rc = LBM_OK;
    for (const Shape &sh : shapes) {
        rc = lbm_batch_set_config(b, sh.block, sh.per_sm, graph);
        if (!rc) rc = lbm_batch_set_launch(b, sh.launch);
        if (!rc) rc = lbm_batch_step(b, steps_per_trial, stream);   // warm-up (and graph capture)
        if (rc) break;
        cudaEventRecord(e0, st);
        rc = lbm_batch_step(b, steps_per_trial, stream);
        if (rc) break;
        cudaEventRecord(e1, st);
        cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) {
            rc = fail(LBM_ERR_CUDA, cudaGetErrorString(e));
            break;
        }
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms / steps_per_trial < best) {
            best = ms / steps_per_trial;
            keep = sh;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    rc = lbm_batch_set_config(b, keep.block, keep.per_sm, graph);
    if (!rc) rc = lbm_batch_set_launch(b, keep.launch);
    if (rc) return rc;
    if (block) *block = keep.block;
    if (blocks_per_sm) *blocks_per_sm = keep.per_sm;
    if (best_ms_per_step) *best_ms_per_step = best;
    return LBM_OK;
}

}  // extern "C"
