// Internal declarations of the iblgf_b200 library (host side).
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <atomic>
#include <cstdint>
#include <functional>
#include <map>
#include <tuple>
#include <unordered_map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/iblgf_b200.h"
#include "keys.hpp"

namespace iblgf_b200
{
struct Error : std::runtime_error
{
    int code;
    Error(int c, const std::string& m)
    : std::runtime_error(m)
    , code(c)
    {
    }
};

#define IBLGF_CUDA(call)                                                                      \
    do                                                                                        \
    {                                                                                         \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            throw ::iblgf_b200::Error(e_ == cudaErrorMemoryAllocation ? IBLGF_ENOMEM : IBLGF_ECUDA, \
                                      std::string(#call) + ": " + cudaGetErrorString(e_));   \
    } while (0)

// Fault injection on the host: when armed (>= 0) the countdown is decremented
// by every device allocation of the library, and the allocation that finds it
// at 0 fails with IBLGF_ENOMEM instead of calling the allocator (then the
// countdown disarms itself). Set through iblgf_debug_fail_alloc().
inline std::atomic<long long>& alloc_fail_countdown()
{
    static std::atomic<long long> v{-1};
    return v;
}
inline void simulated_alloc_failure()
{
    auto& v = alloc_fail_countdown();
    long long cur = v.load();
    while (cur >= 0)
        if (v.compare_exchange_weak(cur, cur - 1))
        {
            if (cur == 0) throw Error(IBLGF_ENOMEM, "simulated device allocation failure (iblgf_debug_fail_alloc)");
            return;
        }
}

// Owning device buffer.
template<class T>
struct DevBuf
{
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept { std::swap(p, o.p), std::swap(n, o.n); }
    DevBuf& operator=(DevBuf&& o) noexcept
    {
        std::swap(p, o.p);
        std::swap(n, o.n);
        return *this;
    }
    ~DevBuf() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count)
    {
        release();
        if (count == 0) return;
        simulated_alloc_failure();
        IBLGF_CUDA(cudaMalloc(&p, count * sizeof(T)));
        n = count;
    }
    void upload(const std::vector<T>& h, cudaStream_t s)
    {
        if (h.size() != n) alloc(h.size());
        if (n) IBLGF_CUDA(cudaMemcpyAsync(p, h.data(), n * sizeof(T), cudaMemcpyHostToDevice, s));
    }
};

// ------------------------------------------------------------- host octree
struct HOct
{
    u64 key = 0;
    int level = 0;
    int parent = -1;
    int child[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
    bool has_data = false;
    int bbase[3] = {0, 0, 0};
    bool leaf = false, correction = false, physical = false;
    int idx = -1;  // canonical position (has_data only)
};

struct HostTree
{
    int e = 0;
    int base_level = 0, depth = 0;
    int base_shift[3] = {0, 0, 0};
    int key_bd_extent[3] = {0, 0, 0};
    std::vector<HOct> o;  // o[0] is the root

    void init(int block_extent, const int* bd_base, const int* bd_extent);
    void add_base_blocks(const std::vector<std::array<int, 3>>& normalized_bases);
    int find(u64 k) const;
    int insert(u64 k);
    int refine_child(int p, int i);
    void alloc(int i, int data_level);
    std::vector<int> dfs_order() const;  // reference depth-first order, root first
    std::vector<u64> unfound_neighbors(int i, bool correction_as_neighbors) const;
    bool try_2to1(u64 k, std::map<u64, bool>& checklist) const;
    void refine(int i, bool ratio_2to1);
    void init_refine(int n_ref, int level_up_max, iblgf_refine_fn pred, void* user);
    // aim_del (per tree position, may be null): deletion marks of an adaptation
    void mark_correction(std::vector<char>* aim_del = nullptr);
    bool leaf_search(int i, bool require_data) const;
    void delete_oct(int i);
    // one adaptation (server side of Domain::adapt): attempts (key, level
    // change) of leaves, ib per tree position (bit 0 is_ib, bit 1 extended);
    // returns the tree positions of the parents whose children take
    // interpolated data, in (level, key) order
    std::vector<int> adapt(const std::vector<std::pair<u64, int>>& attempts, const std::vector<char>& ib,
                           bool& base_mesh_update);
    void import_octants(int n, const u64* keys, const int* flags);
    void restart(int n, const u64* keys, const unsigned char* leaf);
    std::vector<int> canonical() const;  // has_data octants, (level, key) order
};

// ------------------------------------------------------------- FMM plan
struct TpTasks  // tensor-product transfer tasks of one tree level
{
    int n_groups = 0;           // one group per receiving block
    int n_tasks = 0;
    DevBuf<int> group_ptr;      // CSR over tasks
    DevBuf<int> group_dst;      // receiving octant
    DevBuf<int> task_src;       // sending octant
    DevBuf<int> task_cid;       // child id (0..7)
};

// sibling groups per group-MAC tile; the kernel's thread rows x groups per
// row cover exactly this many
constexpr int kGroupTileCap = 32;
// sibling groups per work item of the block-Toeplitz MAC (a tile has up to 3)
constexpr int kToeplitzPart = 14;

struct FmmPlan
{
    int level = 0, mask_idx = 0;
    DevBuf<int> zero_s, zero_t, copy_s, add_t;
    std::vector<TpTasks> antrp;  // levels level-1 .. 0
    std::vector<TpTasks> intrp;  // levels 1 .. level-1
    int n_src = 0, n_tgt = 0;
    DevBuf<int> src_oct;         // source slot -> octant
    DevBuf<int> tgt_oct;         // target slot -> octant
    DevBuf<int> pair_ptr;        // CSR over targets
    DevBuf<int> pair_src;        // source slot
    DevBuf<int> pair_spec;       // spectrum slot
    long long n_pairs = 0;
    int n_spec_unique = 0;
    // targets handled by the general pair-list MAC come first in tgt_oct
    int n_csr_tgt = 0;
    // sibling-group MAC: tiles of groups, staged source lists, per-group
    // candidate sources (216, local index into the tile's staged list, 0xFFFF
    // for none) and targets (8 child slots), LGF spectrum slot per offset
    int n_tiles = 0, max_tile_src = 0, n_groups = 0;
    // tile_jr: per tile kGroupTileCap x 216 source rows of its groups'
    // candidates (the zero row for absent ones)
    DevBuf<int> tile_gptr, tile_jr, tile_tab, tile_coarse, spec_u, grp_tgt;
    DevBuf<unsigned> grp_pm;     // per group: bit n set = neighbour parent n has a candidate
    DevBuf<int> tile_combo;      // per tile: coefficient table of the block-Toeplitz MAC (its level difference)
    DevBuf<int> tile_parts;      // block-Toeplitz work: tile << 2 | part for the non-empty parts of 14 groups
    int n_parts = 0;
    // tensor-core MAC: tiles of up to 128 consecutive groups of one LGF table
    // and pair mode (tc_gptr, tc_tab, tc_mode, tc_pm = union of the groups'
    // parent masks), and per group its 216 candidate source rows (grp_jr)
    int n_tc = 0;
    DevBuf<int> tc_gptr, tc_tab, tc_mode, grp_jr;
    DevBuf<unsigned> tc_pm;
    // neighbour-only plans: the direct separable sweep's targets and their
    // 27 neighbour sources (octants, -1: none)
    int n_ge = 0;
    DevBuf<int> ge_tgt, ge_src;
    long long n_exec = 0;        // (target, source) products the MAC kernels execute
    long long mac_flops = 0;     // floating-point operations of the MAC kernels per frequency
    bool adj_only = false;       // every tile takes adjacent pairs only (integrating factor)
    mutable int mac_variant = -1;  // group-MAC variant chosen by the autotuner (-1: not tuned yet)
    bool empty() const { return n_tgt == 0; }
};

// Host side of a sweep plan: octant indices, source / target slots and LGF
// spectrum keys (level_diff or -1-ge, block offset). upload_plan() maps the
// keys to slots of a context's spectra cache and moves the lists to the
// device; merge_plans() concatenates the plans of independent octrees.
struct HostTasks
{
    std::vector<int> ptr{0}, src, cid, dst;  // receiving blocks with at least one task
};
struct HostPlan
{
    int level = 0, mask_idx = 0, ge = -1;
    std::vector<int> zs, zt, cs, at, srcs;
    std::vector<HostTasks> antrp, intrp;
    std::vector<int> tgt_list;  // pair-list targets first, then group targets
    int n_csr_tgt = 0;
    std::vector<int> ptr{0}, psrc;
    std::vector<std::array<int, 4>> pkey;      // keys of the pair-list (CSR) targets' pairs
    std::vector<std::array<int, 4>> all_keys;  // keys of every target's pairs: spectra to compute
    std::vector<int> tgptr{0}, tsptr{0}, tsrc, ttab, tcoarse, gtgt;
    std::vector<unsigned short> gsrc;
    std::vector<unsigned> gpm;
    // neighbour-only (integrating factor) plans: per target octant its
    // source octants by neighbour offset, (ox+1) + 3 (oy+1) + 9 (oz+1), -1: none
    std::vector<int> ge_tgt, ge_src;
    std::vector<std::array<int, 4>> tab_keys;  // 343 per table
    int n_groups = 0, max_tile_src = 0, n_spec_unique = 0;
    long long n_pairs = 0, n_exec = 0;
};

// Field storage comes from a per-device stream-ordered memory pool that keeps
// freed memory mapped: an adaptation reallocates every field, and plain
// cudaMalloc / cudaFree of that many large buffers costs up to seconds once
// the device has seen other large allocations come and go.
cudaMemPool_t field_pool(int device);
struct PoolBuf
{
    double* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    PoolBuf() = default;
    PoolBuf(const PoolBuf&) = delete;
    PoolBuf& operator=(const PoolBuf&) = delete;
    PoolBuf& operator=(PoolBuf&& o) noexcept
    {
        std::swap(p, o.p);
        std::swap(n, o.n);
        std::swap(s, o.s);
        return *this;
    }
    ~PoolBuf() { release(); }
    void release()
    {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count, int device, cudaStream_t stream)
    {
        release();
        s = stream;
        if (count == 0) return;
        simulated_alloc_failure();
        IBLGF_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p), count * sizeof(double),
                                           field_pool(device), stream));
        n = count;
    }
};

struct Field
{
    PoolBuf d;
};

constexpr int kNumStats = 10;

struct Ctx
{
    iblgf_config cfg{};
    int Nb = 0, P = 0;
    long long NC = 0;  // complex values per half spectrum, Nb * P * P
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;

    HostTree tree;
    std::vector<std::array<int, 3>> pending_bases;
    bool finalized = false;
    bool subtract_non_leaf = false, use_correction = true;

    // canonical octant arrays (host mirrors)
    int n_oct = 0;
    std::vector<u64> keys;
    std::vector<int> levels, flags, bbase, parent, child;  // child: 8 per octant
    std::vector<int> nbr, infl, n_infl;                   // from the device
    std::vector<std::vector<uint8_t>> masks;              // [mask_idx][2*oct]
    std::vector<std::vector<int>> level_octs;             // canonical idx per level
    std::unordered_map<u64, int> key_index;               // key -> canonical idx

    // device octant data
    DevBuf<int> d_bbase, d_nbr;
    // leaf blocks in canonical order and the device staging of their
    // interiors (leaf-interior field transfers); rebuilt with the domain
    DevBuf<int> d_leaf_blocks;
    int n_leaf_blocks = -1;
    PoolBuf leaf_stage;
    // asynchronous leaf downloads: gathered into leaf_out on `stream`, copied
    // to the host on copy_stream (created on first use)
    PoolBuf leaf_out;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_gathered = nullptr, ev_copied = nullptr;
    // asynchronous leaf uploads: host -> leaf_in on copy_stream, scattered
    // into the field on `stream` (which waits for the copy); the next copy
    // into leaf_in waits for the scatter
    PoolBuf leaf_in;
    cudaEvent_t ev_in_copied = nullptr, ev_scattered = nullptr;

    // fields
    std::vector<std::unique_ptr<Field>> fields;
    int f_source_tmp = -1, f_target_tmp = -1, f_correction_tmp = -1, f_fmm_s = -1, f_fmm_t = -1;

    // LGF table (device), twiddles, transfer matrices
    DevBuf<double> d_lgf_table;
    DevBuf<double> d_tw64;  // 2P doubles: cos, -sin interleaved (forward)
    // Nb*Nb matrices (child bit 0 / 1): [0,1] FMM Nli, cell-centred transfers with
    // relative position 1: [2,3] interpolation, [4,5] coarsification; relative
    // position 0: [6,7] interpolation, [8,9] coarsification (injection)
    DevBuf<double> d_mats;
    std::vector<double> h_mats;  // host copy (transfer kernels take them as launch parameters)

    // spectra cache: key (level_diff, bx, by, bz) -> slot; storage in the
    // working precision, NC complex per slot
    std::map<std::array<int, 4>, int> spec_slot;
    int spec_cap = 0, spec_used = 0;
    DevBuf<char> d_spec;

    // per-sweep work buffers (sized on demand)
    DevBuf<char> d_src_spec, d_acc, d_w;

    // coefficient tables of the block-Toeplitz group MAC, one per level
    // difference: 729 rows of NC complex (working precision) each, and the
    // TMA tensor map (CUtensorMap, 128 bytes) over all of them
    std::map<int, int> combo_of_ld;
    int combo_tables = 0, combo_cap = 0;
    DevBuf<char> d_combo;
    alignas(64) unsigned char combo_map[128] = {};

    std::map<std::tuple<int, int, int>, std::unique_ptr<FmmPlan>> plans;
    // integrating-factor kernels: e^{-2 alpha} I_n(2 alpha), n < ge_stride, one
    // table per alpha (LGF_GE::build_lt / compute_lgf)
    std::map<double, int> ge_index;
    std::vector<double> ge_host;
    DevBuf<double> d_ge;
    int ge_stride = 0;
    long long launches = 0;
    // group-MAC autotuning: a variant pinned by the caller (-1: tune per
    // plan) and one record per tuned plan: level, mask index, targets, ms of
    // variants 0, 1, 2, 3 (-1: not applicable), chosen variant
    int mac_variant_forced = -1;
    // integrating-factor sweeps by direct separable sums when the kernel allows
    bool ge_direct_enabled = true;
    bool trace = false;  // IBLGF_TRACE: plan-build trace lines on stderr
    std::vector<std::array<double, 8>> mac_tuning;
    // the autotuner's choice per (tree level, mask index), reused by plans
    // rebuilt for the same sweep after an adaptation instead of re-timing
    std::map<std::pair<int, int>, int> mac_choice;
    // device status word: bounded waits in kernels that run out set bits
    // (kStatusTimeout); read and cleared by check_status()
    DevBuf<int> d_status;
    bool profile = false;
    std::vector<std::array<cudaEvent_t, 5>> prof_events;
    // work counters since the last reset: sweeps, sources, targets, pairs,
    // unique spectra per sweep, anterpolation tasks, interpolation tasks
    // sweeps, sources, targets, pairs, unique spectra, anterp tasks, interp
    // tasks, group-MAC targets, MAC products executed
    long long stats[kNumStats] = {};

    // sharded sweeps (one rank of several): owner rank per canonical octant
    // (empty: not sharded); a sweep computes the targets this rank owns (and
    // the coarser targets their values are interpolated from), then the
    // exchange callback sums the sweep's level targets over the ranks
    std::vector<int> owner;
    int rank = 0;
    iblgf_exchange_fn exchange_fn = nullptr;
    void* exchange_user = nullptr;
    PoolBuf exchange_buf;

    // batch of independent problems (iblgf_batch_*): each problem's octree,
    // lists and masks live in a topology-only sub-context; fields, spectra and
    // work buffers live here, the problems' octants back to back
    bool batch = false, topology_only = false, has_blocks = false;
    std::vector<std::unique_ptr<Ctx>> sub;
    std::vector<int> sub_off;

    // per-context state of the other modules (batch lists and plans,
    // immersed boundary, time stepping, level lists), created on first use
    // and owned here, so that contexts driven from different host threads
    // share no mutable state
    enum { kExtBatch, kExtIb, kExtNsOpt, kExtNs, kExtNsPending, kExtPLists, kExtOpLists, kNumExt };
    std::shared_ptr<void> ext[kNumExt];
    template<class T>
    T* ext_get(int i) const
    {
        return static_cast<T*>(ext[i].get());
    }

    size_t block_elems() const { return (size_t)Nb * Nb * Nb; }
    size_t field_elems() const { return (size_t)n_oct * block_elems(); }
    size_t cplx_bytes() const { return cfg.precision == IBLGF_FP32 ? 8 : 16; }
    double* field(int id) { return fields.at(id)->d.p; }
};

// -------------------------------------------------------------- library
void ctx_init(Ctx& c);
void domain_finalize(Ctx& c);
int field_create(Ctx& c);
void fmm_apply(Ctx& c, int src, int tgt, int level, bool nlas, double scale, int fmm_type, int ge = -1);
// one FMM sweep of a ready plan: zero / copy / anterpolate, forward transforms,
// MAC, inverse transforms + add, interpolate, add into tgt (fmm.hpp:729-870)
void run_sweep(Ctx& c, FmmPlan& p, int src, int tgt, double dx_level, double add_with_scale, int ge);
// direct_only: a neighbour-only plan for the direct separable sweep (target
// and neighbour lists only; no pair lists, groups or spectra)
HostPlan build_host_plan(const Ctx& c, int level, int idx, int ge, bool direct_only = false);
void prebuild_plans(Ctx& c, const std::vector<std::tuple<int, int, int>>& keys);
std::unique_ptr<FmmPlan> upload_plan(Ctx& c, const HostPlan& h);
void host_tasks(HostTasks& ht, const std::vector<int>& dst, const std::vector<std::vector<std::pair<int, int>>>& tasks);
void upload_host_tasks(Ctx& c, TpTasks& tt, const HostTasks& ht);
void add_blocks(Ctx& c, int n, const int* base, const int* extent);
void need_single(const Ctx& c);
// batches of independent problems (batch.cpp)
int batch_add_problem(Ctx& c, const int* bd_base, const int* bd_extent, int n, const int* base, const int* extent,
                      int n_ref, iblgf_refine_fn pred, void* user);
void batch_finalize(Ctx& c);
void batch_apply_lgf(Ctx& c, int src, int tgt);
void batch_release(Ctx& c);
// immersed boundary (ibsolve.cpp)
void build_ib_masks(Ctx& c, std::vector<int>& ib);
void ib_set_points(Ctx& c, int n, const double* X, double Re);
// false when the solve stopped at max_iter without converging (f and iters
// are written either way)
bool ib_solve(Ctx& c, const int* u, double alpha, double threshold, int max_iter, double* f, int* iters);
// IB steps can be captured in a graph (the learned warm start reads the host)
bool ib_graphable(const Ctx& c);
void ib_flags(Ctx& c, int* flags);
bool ib_active(const Ctx& c);
const int* ib_face_aux2(Ctx& c);
// write_prev = false (the velocity-refresh correction stages): the CG starts
// from the stage's previous force but the result does not replace it, and the
// learned warm start neither predicts nor records samples
void ns_ib_stage(Ctx& c, int stage, double alpha, double threshold, int max_iter, int d_field, const int* face_aux,
                 const std::function<void()>& gradient_d, bool write_prev = true);
void ib_force(Ctx& c, int stage, double* out, int* iters, int* not_converged = nullptr);
void ib_release(Ctx& c);
void launch_ib_projection(Ctx& c, const double* const* u, const int* ptr, const long long* at, const double* w,
                          int n, double* f);
void launch_ib_smearing(Ctx& c, double* const* u, const long long* node_at, const int* nptr, const int* npt,
                        const int* nent, const double* w, int n_nodes, const double* f);
void launch_face_planes(Ctx& c, double* f, const int* list, const unsigned char* faces, int n, int width);
// device force CG (ib.cu): FP64 dot products by one CTA in a fixed order;
// ctl = [done, iterations, not converged], sc = [rsold, p.Ap, rsnew, f.f]
void launch_cg_dot(Ctx& c, const double* a, const double* b, const double* a2, const double* b2, int n,
                   double* out0, double* out1, const int* ctl);
void launch_cg_init(Ctx& c, const double* uc, const double* Ax, double* r, double* p, int n, int* ctl, int max_iter);
void launch_cg_update(Ctx& c, double* f, double* r, const double* p, const double* Ap, int n, const double* sc,
                      int* ctl);
void launch_cg_direction(Ctx& c, double* p, const double* r, int n, const double* sc, const int* ctl,
                         double threshold);
void launch_cg_advance(Ctx& c, double* sc, int* ctl, double threshold, int max_iter, unsigned long long cond,
                       bool set_cond);
void launch_cg_record(Ctx& c, const int* ctl, int* rec);
// CG warm start (ib.cu): f0 = f_prev, or 2 f_prev - f_prev2 once count >= 2
// when extrapolating; record shifts the stage's force history
void launch_ws_base(Ctx& c, double* f0, const double* fp, const double* fp2, int n, const int* count, bool extrapolate);
void launch_ws_record(Ctx& c, double* fp2, double* fp, const double* f, int n, int* count);
// learned warm start network (warmstart.cu)
constexpr int kWsChannels = 64, kWsInputs = 9;
void ws_offsets(int* off);  // 7 offsets: W1 b1 W2 b2 W3 b3 end
void ws_forward(Ctx& c, const float* params, const float* x, int S, int N, float* h1, float* h2, float* y);
float ws_backward(Ctx& c, const float* params, const float* x, const float* tgt, int S, int N, const float* h1,
                  const float* h2, const float* y, float* dy, float* dh2, float* dh1, float* grads,
                  DevBuf<float>& partial);
void ws_adam(Ctx& c, float* params, const float* grads, float* m, float* v, int n, float lr, int step);
void ib_warmstart(Ctx& c, int mode, int train_steps, int epochs, double lr, unsigned seed);
void ib_warmstart_info(Ctx& c, double* info);
void ws_check(Ctx& c, int S, int N, const float* params, const float* x, const float* tgt, float* y, float* grads,
              float* loss);
int ge_table(Ctx& c, double alpha);
// rp: relative position per axis of the field's mesh object (cell {1,1,1} when null)
void apply_if(Ctx& c, int src, int tgt, double alpha_base, int fmm_type, const int* rp = nullptr);

// device block lists of the Poisson level loop and of the level-wise operators
struct PoissonLists
{
    DevBuf<int> all, leaves;
    std::vector<DevBuf<int>> level_all, level_leaves;
    std::vector<TpTasks> coarsify;       // per level ls (dst parents at ls)
    std::vector<TpTasks> cc_intrp;       // per level l: children of level-l octants
    std::vector<TpTasks> corr_intrp;     // per level l: correction children
    std::vector<DevBuf<int>> children;   // per level l: children (with data) of level-l octants
};
struct OpLists
{
    std::vector<DevBuf<int>> list;
    std::vector<DevBuf<double>> dx;
};
PoissonLists& poisson_lists(Ctx& c);
// IF-HERK time steps (ifherk.hpp:1078-1200) of the face velocity u[3] and the
// cell pressure p; T advances by dt per step
void ns_step(Ctx& c, const int* u, int p, double dt, double Re, double* T, int n_steps);
// constant frame velocity and IB CG settings of the IF-HERK step
void ns_options(Ctx& c, const double* frame_vel, double cg_threshold, int cg_max_iter);
void ns_release(Ctx& c);
// after an adaptation: the time step's per-tree lists are rebuilt, its graph
// dropped; base_mesh_update forces a velocity refresh at the next step
void ns_on_adapt(Ctx& c, bool base_mesh_update, const std::vector<char>& old_corr);
// Ifherk's scratch fields read by the adapt condition: cell_aux, edge_aux[3],
// correction_tmp of the Poisson solver
void ns_fields(Ctx& c, int* ids);
void ns_clean(Ctx& c, int field, bool non_leaf_only, int width);
void ns_clean_leaf_correction_boundary(Ctx& c, const int* fields, int n, int level, bool leaf_only_boundary);
void ib_on_adapt(Ctx& c);
// per-octant IB flags (bit 0 is_ib, bit 1 is_extended_ib); empty without IB
std::vector<int> ib_octant_flags(Ctx& c);
// octree rebuild after the host tree changed (lists, masks; no fields)
void domain_rebuild(Ctx& c);
// Ifherk::adapt + Domain::adapt for one process: attempts (key, level change),
// then every field remapped to the new octants, the listed fields
// interpolated into the children of the interpolation parents
void domain_adapt(Ctx& c, int n_att, const u64* keys, const int* lchange, int n_interp, const int* interp_fields,
                  const int* interp_mesh, int* base_mesh_update);
void block_norms(Ctx& c, const int* fields, int n_comp, double* host_max, double* host_rms);
OpLists& op_lists(Ctx& c);
void apply_op_octants(Ctx& c, int op, const int* in, int n_in, const int* out, int n_out, const int* octants, int n,
                      double scale);
void poisson_apply_lgf(Ctx& c, int src, int tgt, int fmm_type);
int mask_idx_gen(int type, int refinement_level, int nlas);

// -------------------------------------------------------------- kernels (.cu)
void launch_lgf_table(Ctx& c);
void launch_lgf_eval(Ctx& c, const int* d_coords, size_t n, double* d_out);
void launch_lgf_ge_eval(Ctx& c, int ge, const int* d_coords, size_t n, double* d_out);
void launch_build_lists(Ctx& c, const u64* d_sorted_keys, const int* d_sorted_idx, int n_sorted,
                        const u64* d_keys, int n, int* d_nbr, int* d_infl, int* d_ninfl);
void launch_spectra(Ctx& c, const std::vector<std::array<int, 5>>& new_slots);
void launch_forward_sources(Ctx& c, const double* fmm_s, const int* d_src_oct, int n_src, void* src_spec);
void launch_mac(Ctx& c, const FmmPlan& p, const void* src_spec, void* acc);
// sibling-group MAC with the fast block-Toeplitz product (group_mac.cu);
// false when the plan's tiles need the direct kernel (adjacent pairs only)
bool toeplitz_mac(Ctx& c, const FmmPlan& p, const void* src_spec, void* acc);
// the coefficient table of level difference ld from the 343 spectrum slots
// of its offsets (created once per context)
int combo_table(Ctx& c, int ld, const std::vector<int>& slots);
// direct separable sweep of a neighbour-only plan with integrating-factor
// table ge (adds into ft); false if the plan or the table does not allow it
bool ge_direct_ok(const Ctx& c, int ge);
bool launch_ge_direct(Ctx& c, const FmmPlan& p, const double* fs, double* ft, int ge, double scale);
// tensor-core sibling-group MAC (FP32 path); false if not applicable
bool tc_mac_ok(const Ctx& c, const FmmPlan& p);
bool tc_mac(Ctx& c, const FmmPlan& p, const void* src_spec, void* acc);
// tensor-core tiles from the CUDA-core tiles (tile group ranges, tables and
// modes) and the groups' parent masks
void build_tc_tiles(const std::vector<int>& tgptr, const std::vector<int>& ttab, const std::vector<int>& tmode,
                    const std::vector<unsigned>& gpm, std::vector<int>& gptr, std::vector<int>& tab,
                    std::vector<int>& mode, std::vector<unsigned>& pm);
// waits for the context stream and throws IBLGF_ETIMEOUT if a kernel's
// bounded wait ran out since the last check
void check_status(Ctx& c);
void launch_inverse_add(Ctx& c, const FmmPlan& p, const void* acc, double* fmm_t, double scale);
// prime-factor inverse (inverse.cu); false when the block size has no
// prime-factor split (the direct inverse runs instead)
bool inverse_pfa(Ctx& c, const void* acc, const int* d_tgt_oct, int n, double scale, double* target,
                 bool fp32_passes);
void init_pfa_constants(int device);
// sharding (solver.cpp): the reference server's load-balanced partition and
// this context's share of it
std::vector<int> domain_partition(const Ctx& c, int n);
void domain_set_owner(Ctx& c, const int* owner, int rank, iblgf_exchange_fn fn, void* user);
// whether the prime-factor inverse runs its z and y passes in FP32
bool inverse_fp32_passes(const Ctx& c);
void launch_zero_blocks(Ctx& c, double* f, const int* list, int n);
void launch_fill_zero(Ctx& c, double* p, size_t n);
void launch_remap_blocks(Ctx& c, const double* old, double* nw, const int* d_src, int n_new);
void launch_block_norms(Ctx& c, const double* const* comps, int n_comp, double* d_max, double* d_rms);
// leaf-interior transfers: staging [leaf][e^3] (x fastest) <-> field blocks
void launch_leaves_scatter(Ctx& c, const double* stage, double* field, const int* list, int n);
void launch_leaves_gather(Ctx& c, const double* field, double* stage, const int* list, int n);
// whole blocks of the listed octants <-> a contiguous buffer [n][Nb^3]
void launch_blocks_gather(Ctx& c, const double* field, double* buf, const int* list, int n);
void launch_blocks_scatter(Ctx& c, const double* buf, double* field, const int* list, int n);
void field_upload_leaves(Ctx& c, int f, const double* host, size_t count);
void field_download_leaves(Ctx& c, int f, double* host, size_t count);
void field_download_leaves_async(Ctx& c, int f, double* host, size_t count);
void copy_stream_release(Ctx& c);
void field_upload_leaves_async(Ctx& c, int f, const double* host, size_t count);
void launch_copy_interior(Ctx& c, const double* src, double* dst, const int* list, int n);
void launch_axpy_blocks(Ctx& c, const double* src, double* dst, const int* list, int n, double a,
                        bool assign);
// fp32: the three passes in FP32, the sum into the FP64 receiving block in FP64
void launch_tp(Ctx& c, const TpTasks& t, const double* src, double* dst, int mat_base,
               int mode /*0 antrp add, 1 intrp add, 2 intrp assign*/, bool fp32 = false);
// per-axis matrix pairs (mat_base[3]): face / edge components of the cell-centred transfers
void launch_tp_axes(Ctx& c, const TpTasks& t, const double* src, double* dst, const int* mat_base, int mode,
                    bool fp32 = false);
void launch_halo(Ctx& c, double* f, const int* list, int n);
void launch_source_correction(Ctx& c, const double* target_tmp, double* corr, const int* list, int n,
                              double inv_dx2);
void launch_op(Ctx& c, int op, const double* const* in, int n_in, double* const* out, int n_out, const int* list,
               const double* dx, int n, double scale);
void buffer_exchange(Ctx& c, int field, int level);
void apply_op(Ctx& c, int op, const int* in, int n_in, const int* out, int n_out, int level, double scale);
void launch_conv_block(Ctx& c, const double* src, const double* kernel, double* out, double scale);
void launch_conv_block_noalloc(Ctx& c, const double* src, const double* kernel, double* out, double scale);

}  // namespace iblgf_b200
