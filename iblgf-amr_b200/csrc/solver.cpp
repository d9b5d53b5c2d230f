// Host driver of the B200 LGF-FMM path: context set-up, domain finalisation
// (device list build, FMM masks), FMM sweep plans and the Poisson level loop.
//
//   FmmMaskBuilder (include/iblgf/fmm/fmm.hpp:54-681): fmm_dry_init_base_level_
//     masks, fmm_upward_pass_masks, fmm_clean_no_inf_masks, stream mask
//   Fmm::apply (fmm.hpp:729-870): one plan per (mask index, level) with the
//     zero/copy lists, per-level anterpolation and interpolation task lists,
//     and the (target, source, LGF spectrum) pair list of all targets of all
//     levels; executed as one batched sweep on the device
//   PoissonSolver::apply_lgf (solver/poisson/poisson.hpp:587-894)
//
// All device work is ordered on the context stream; a sweep issues no host
// synchronisation once its plan exists.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>

#include "ctx.hpp"

namespace iblgf_b200
{
bool nb_supported(int Nb);
void init_twiddle_constants(int device);

int mask_idx_gen(int type, int refinement_level, int nlas)
{
    if (type == IBLGF_STREAM) return 0;
    if (type == IBLGF_AMR2AMR) return refinement_level * 2 + nlas + 15;
    if (type == IBLGF_IB2xIB) return 1;
    if (type == IBLGF_xIB2IB) return 2;
    if (type == IBLGF_IB2AMR) return refinement_level + 4;
    throw Error(IBLGF_EINVAL, "unsupported fmm_type");
}

// --------------------------------------------------------------- matrices
namespace
{
// Lagrange node-transfer matrix, Nb x 2Nb with (p, c) at p*2Nb + c:
// fmm_nli.hpp:319-374 (relpos 0, integer offsets) and
// cell_center_nli_intrp.hpp:677-787 (relpos 1, half-cell offsets)
std::vector<double> lagrange_matrix(int Nb, int pts_cap, int relpos)
{
    std::vector<double> m((size_t)Nb * 2 * Nb, 0.0);
    auto M = [&](int p, int c) -> double& { return m[(size_t)p * 2 * Nb + c]; };
    for (int c = 1; c < 2 * Nb - 1; ++c)
    {
        if (relpos == 0 && c % 2 == 0)
        {
            M(c / 2, c - 1) = 1.0;
            continue;
        }
        const double cp = relpos == 0 ? (double)(c - Nb) : c - Nb + 0.5;
        int bl, br;
        if (cp < -1)
        {
            bl = std::max(0, (c + 1) / 2 - pts_cap / 2);
            br = std::min(Nb, bl + pts_cap);
        }
        else
        {
            br = std::min(Nb, (c + 1) / 2 + pts_cap / 2);
            bl = std::max(0, br - pts_cap);
        }
        long double sum = 0.0;
        for (int p = bl; p < br; ++p)
        {
            long double w = 1.0;
            const int pp = 2 * p - Nb + 1;
            for (int l = bl; l < br; ++l)
                if (l != p) w /= -(long double)(2 * l - Nb + 1 - pp);
            w /= relpos == 0 ? (long double)((int)cp - pp + 1) : (long double)(cp - pp);
            M(p, c - 1) = (double)w;
            sum += w;
        }
        for (int p = 0; p < Nb; ++p) M(p, c - 1) /= (double)sum;
    }
    for (int c = 2 * Nb - 1; c > Nb - 1; --c)
        for (int p = 0; p < Nb; ++p) M(p, c) = M(p, c - 2);
    return m;
}

void append_halves(std::vector<double>& out, const std::vector<double>& full, int Nb)
{
    for (int h = 0; h < 2; ++h)
        for (int p = 0; p < Nb; ++p)
            for (int j = 0; j < Nb; ++j) out.push_back(full[(size_t)p * 2 * Nb + h * Nb + j]);
}
}  // namespace

void ctx_init(Ctx& c)
{
    // IBLGF_TRACE=1: one stderr line per FMM plan build (host build and
    // upload times) for tracing set-up and adaptation costs
    const char* tr = std::getenv("IBLGF_TRACE");
    c.trace = tr && tr[0] && tr[0] != '0';
    const int e = c.cfg.block_extent;
    c.Nb = e + 2;
    c.P = 2 * c.Nb - 1;
    c.NC = (long long)c.Nb * c.P * c.P;
    if (!nb_supported(c.Nb)) throw Error(IBLGF_EINVAL, "unsupported block_extent (supported: 4,6,8,10,14,16)");
    if (c.cfg.precision != IBLGF_FP64 && c.cfg.precision != IBLGF_FP32)
        throw Error(IBLGF_EINVAL, "precision must be IBLGF_FP64 or IBLGF_FP32");
    if (c.cfg.intrp_order <= 0) c.cfg.intrp_order = 5;
    IBLGF_CUDA(cudaSetDevice(c.cfg.device));
    if (c.cfg.stream) c.stream = (cudaStream_t)c.cfg.stream;
    else
    {
        IBLGF_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
        c.own_stream = true;
    }
    if (c.topology_only)
    {
        c.tree.init(e, c.cfg.bd_base, c.cfg.bd_extent);
        return;
    }
    c.d_status.alloc(1);
    IBLGF_CUDA(cudaMemsetAsync(c.d_status.p, 0, sizeof(int), c.stream));
    init_twiddle_constants(c.cfg.device);
    init_pfa_constants(c.cfg.device);
    // twiddles e^{-2 pi i j / P}
    std::vector<double> tw(2 * c.P);
    for (int j = 0; j < c.P; ++j)
    {
        const double a = 2.0 * M_PI * j / c.P;
        tw[2 * j] = std::cos(a);
        tw[2 * j + 1] = -std::sin(a);
    }
    c.d_tw64.upload(tw, c.stream);
    // [0,1] FMM Nli (pts_cap 10), [2,3] cell-centred interpolation (relpos 1),
    // [4,5] cell-centred coarsification (2-point average per axis)
    std::vector<double> mats;
    append_halves(mats, lagrange_matrix(c.Nb, 10, 0), c.Nb);
    append_halves(mats, lagrange_matrix(c.Nb, c.cfg.intrp_order, 1), c.Nb);
    std::vector<double> simple((size_t)c.Nb * c.Nb * 2, 0.0);
    for (int h = 0; h < 2; ++h)
        for (int p = 1; p < c.Nb - 1; ++p)
            for (int j = 1; j < c.Nb - 1; ++j)
            {
                const int col = j + h * (c.Nb - 2);  // column of the Nb x (2Nb-2) averaging matrix
                if (col == 2 * p - 1 || col == 2 * p) simple[(size_t)h * c.Nb * c.Nb + p * c.Nb + j] = 0.5;
            }
    mats.insert(mats.end(), simple.begin(), simple.end());
    // relative position 0 (face normal / edge transverse axes): Lagrange
    // interpolation on coincident nodes, injection for coarsification
    // (cell_center_nli_intrp.hpp:82-83, 109-118, 158-161)
    append_halves(mats, lagrange_matrix(c.Nb, c.cfg.intrp_order, 0), c.Nb);
    std::vector<double> inject((size_t)c.Nb * c.Nb * 2, 0.0);
    for (int h = 0; h < 2; ++h)
        for (int p = 1; p < c.Nb - 1; ++p)
            for (int j = 1; j < c.Nb - 1; ++j)
                if (j + h * (c.Nb - 2) == 2 * p - 1) inject[(size_t)h * c.Nb * c.Nb + p * c.Nb + j] = 1.0;
    mats.insert(mats.end(), inject.begin(), inject.end());
    c.d_mats.upload(mats, c.stream);
    c.h_mats = mats;
    c.tree.init(e, c.cfg.bd_base, c.cfg.bd_extent);
    launch_lgf_table(c);
}

// The FP32 path runs the prime-factor z and y inverse passes in FP32 (the
// c2r stage, the sum over the two kx halves and the add into the target stay
// FP64). Measured on the 3-level Gaussian workload: 4.8e-6 relative L-inf
// against the FP64 oracle (FP64 passes: 1.4e-7; the direct 35-term FP32 sums
// gave 1.16e-5), inverse phase 1.89 ms instead of 2.53 ms per solve.
// Server::compute_distribution (decomposition/server.hpp:245-330) for this
// process's octree: loads as FmmMaskBuilder::fmm_dry accumulates them
// (fmm.hpp:597-626: neighbour + influence count per AMR2AMR sweep in which
// the octant is a target), then per level from the finest the leaf and
// correction octants in Morton order split into n contiguous runs by
// cumulative load (zero loads count 1), each other octant to the rank of its
// least-loaded child.
std::vector<int> domain_partition(const Ctx& c, int n)
{
    if (!c.finalized) throw Error(IBLGF_EINVAL, "domain not finalized");
    if (n < 1) throw Error(IBLGF_EINVAL, "need at least one rank");
    std::vector<double> load(c.n_oct, 0.0);
    const int depth = c.tree.depth, bl = c.tree.base_level;
    for (int rl = 0; rl < depth - bl; ++rl)
        for (int nlas = 0; nlas < 2; ++nlas)
        {
            const int idx = mask_idx_gen(IBLGF_AMR2AMR, rl, nlas);
            if (idx >= (int)c.masks.size() || c.masks[idx].empty()) continue;
            for (int o = 0; o < c.n_oct; ++o)
            {
                if (!c.masks[idx][2 * o + 1]) continue;
                int nn = 0;
                for (int i = 0; i < 27; ++i) nn += c.nbr[27 * o + i] >= 0 ? 1 : 0;
                load[o] += nn + c.n_infl[o];
            }
        }
    std::vector<int> owner(c.n_oct, -1);
    std::vector<double> total(n, 0.0);
    for (int l = (int)c.level_octs.size() - 1; l >= 0; --l)
    {
        const std::vector<int>& lo = c.level_octs[l];
        auto candidate = [&](int o) { return (c.flags[o] & 3) != 0; };
        double tl = 0.0;
        for (int o : lo)
            if (candidate(o))
            {
                if (load[o] == 0.0) load[o] = 1.0;
                tl += load[o];
            }
        size_t it = 0;
        double cur = 0.0;
        for (int r = 0; r < n && it < lo.size(); ++r)
        {
            const double target = std::min((double)(r + 1) / n * tl, tl);
            int count = 0;
            while (it < lo.size() && (cur <= target || count == 0))
            {
                const int o = lo[it++];
                if (!candidate(o)) continue;
                owner[o] = r;
                total[r] += load[o];
                cur += load[o];
                ++count;
            }
        }
        for (int o : lo)
        {
            if (candidate(o) && owner[o] >= 0) continue;
            int best = -1;
            double bl_load = 0.0;
            for (int k = 0; k < 8; ++k)
            {
                const int ch = c.child[8 * o + k];
                if (ch < 0 || owner[ch] < 0) continue;
                if (best < 0 || total[owner[ch]] < bl_load)
                {
                    best = owner[ch];
                    bl_load = total[owner[ch]];
                }
            }
            if (best >= 0)
            {
                if (owner[o] >= 0) total[owner[o]] -= load[o];
                owner[o] = best;
                total[best] += load[o];
            }
        }
    }
    for (int& w : owner)
        if (w < 0) w = 0;  // octants with neither a leaf role nor children (none in a valid octree)
    return owner;
}

void domain_set_owner(Ctx& c, const int* owner, int rank, iblgf_exchange_fn fn, void* user)
{
    need_single(c);
    if (!c.finalized) throw Error(IBLGF_EINVAL, "domain not finalized");
    if (owner)
    {
        if (!fn) throw Error(IBLGF_EINVAL, "a sharded context needs an exchange callback");
        c.owner.assign(owner, owner + c.n_oct);
        c.rank = rank;
    }
    else
        c.owner.clear();
    c.exchange_fn = fn;
    c.exchange_user = user;
    c.plans.clear();
}

bool inverse_fp32_passes(const Ctx& c) { return c.cfg.precision == IBLGF_FP32; }

void check_status(Ctx& c)
{
    if (!c.d_status.p) return;
    int h = 0;
    IBLGF_CUDA(cudaMemcpyAsync(&h, c.d_status.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    if (!h) return;
    IBLGF_CUDA(cudaMemsetAsync(c.d_status.p, 0, sizeof(int), c.stream));
    if (h & 1) throw Error(IBLGF_ETIMEOUT, "a bounded device wait ran out (results of the affected launches are void)");
    throw Error(IBLGF_EINTERNAL, "device status " + std::to_string(h));
}

// --------------------------------------------------------------- domain
namespace
{
struct MaskView
{
    std::vector<uint8_t>& m;
    bool S(int o) const { return m[2 * o]; }
    bool T(int o) const { return m[2 * o + 1]; }
    void set(int o, bool s, bool t)
    {
        m[2 * o] = s;
        m[2 * o + 1] = t;
    }
};

void upward_pass(Ctx& c, int base_level, MaskView mv)
{
    for (int level = base_level - 1; level >= 0; --level)
    {
        for (int o : c.level_octs[level])
        {
            bool s = false, t = false;
            for (int k = 0; k < 8; ++k)
            {
                const int ch = c.child[8 * o + k];
                if (ch < 0) continue;
                s = s || mv.S(ch);
                t = t || mv.T(ch);
            }
            mv.set(o, s, t);
        }
    }
}

void clean_no_inf(Ctx& c, int base_level, MaskView mv)
{
    for (int level = 0; level < base_level; ++level)
        for (int o : c.level_octs[level])
        {
            const int p = c.parent[o];
            if (mv.S(o))
            {
                if (p >= 0 && mv.S(p)) continue;
                bool has = false;
                for (int i = 0; i < c.n_infl[o] && !has; ++i)
                {
                    const int n = c.infl[189 * o + i];
                    has = n >= 0 && mv.T(n);
                }
                if (!has) mv.m[2 * o] = 0;
            }
            if (mv.T(o))
            {
                if (p >= 0 && mv.T(p)) continue;
                bool has = false;
                for (int i = 0; i < c.n_infl[o] && !has; ++i)
                {
                    const int n = c.infl[189 * o + i];
                    has = n >= 0 && mv.S(n);
                }
                if (!has) mv.m[2 * o + 1] = 0;
            }
        }
}

void build_masks(Ctx& c)
{
    c.masks.assign(50, std::vector<uint8_t>(2 * (size_t)c.n_oct, 0));
    const int bl = c.tree.base_level;
    for (int l = bl; l < c.tree.depth; ++l)
    {
        for (int nlas = 0; nlas <= 1; ++nlas)
        {
            const int idx = mask_idx_gen(IBLGF_AMR2AMR, l - bl, nlas);
            MaskView mv{c.masks[idx]};
            for (int o : c.level_octs[l])
            {
                const bool leaf = c.flags[o] & 1, corr = c.flags[o] & 2;
                bool corr_parent = false;
                for (int k = 0; k < 8; ++k)
                {
                    const int ch = c.child[8 * o + k];
                    if (ch >= 0 && (c.flags[ch] & 2)) corr_parent = true;
                }
                if (nlas)
                {
                    if (c.subtract_non_leaf) mv.set(o, !(leaf || corr), (leaf || corr) ? corr_parent : true);
                    else mv.set(o, leaf || corr, (leaf || corr) ? leaf : true);
                }
                else
                {
                    if (c.subtract_non_leaf) mv.set(o, true, true);
                    else mv.set(o, !(leaf || corr), (leaf || corr) ? leaf : false);
                }
            }
            upward_pass(c, l, mv);
            clean_no_inf(c, l, mv);
        }
    }
    MaskView st{c.masks[mask_idx_gen(IBLGF_STREAM, 0, 0)]};
    for (int o : c.level_octs[bl]) st.set(o, !(c.flags[o] & 2), true);
    upward_pass(c, bl, st);
}
}  // namespace

// FmmMaskBuilder::fmm_IB2xIB_mask / fmm_xIB2IB_mask / fmm_IB2AMR_mask
// (fmm.hpp:70-190) from per-octant flags (bit0 is_ib, bit1 is_extended_ib);
// IB2AMR marks the parents of IB blocks as IB (flags updated in place)
void build_ib_masks(Ctx& c, std::vector<int>& ib)
{
    const int l = c.tree.depth - 1, bl = c.tree.base_level;
    for (int t = IBLGF_IB2xIB; t <= IBLGF_xIB2IB; ++t)
    {
        MaskView mv{c.masks[mask_idx_gen(t, 0, 0)]};
        std::fill(mv.m.begin(), mv.m.end(), 0);
        for (int o : c.level_octs[l])
        {
            if (ib[o] & 1) mv.set(o, true, true);
            if (ib[o] & 2)
            {
                if (t == IBLGF_IB2xIB) mv.m[2 * o + 1] = 1;
                else mv.m[2 * o] = 1;
            }
        }
        upward_pass(c, l, mv);
        clean_no_inf(c, l, mv);
    }
    for (int lv = l - 1; lv >= bl; --lv)
        for (int o : c.level_octs[lv])
            for (int k = 0; k < 8; ++k)
            {
                const int ch = c.child[8 * o + k];
                if (ch >= 0 && (ib[ch] & 1)) ib[o] |= 1;
            }
    for (int lv = l; lv >= bl; --lv)
    {
        MaskView mv{c.masks[mask_idx_gen(IBLGF_IB2AMR, lv - bl, 0)]};
        std::fill(mv.m.begin(), mv.m.end(), 0);
        for (int o : c.level_octs[lv]) mv.set(o, (ib[o] & 1) != 0, true);
        upward_pass(c, lv, mv);
    }
    // plans built from the previous masks are stale
    for (auto it = c.plans.begin(); it != c.plans.end();)
    {
        const int idx = std::get<0>(it->first);
        if (idx >= 1 && idx < 15) it = c.plans.erase(it);
        else ++it;
    }
}

cudaMemPool_t field_pool(int device)
{
    static std::mutex m;
    static std::map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lock(m);
    auto it = pools.find(device);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool;
    IBLGF_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = ~0ull;  // never hand freed memory back while the process runs
    IBLGF_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    pools.emplace(device, pool);
    return pool;
}

int field_create(Ctx& c)
{
    auto f = std::make_unique<Field>();
    f->d.alloc(c.field_elems(), c.cfg.device, c.stream);
    IBLGF_CUDA(cudaMemsetAsync(f->d.p, 0, c.field_elems() * sizeof(double), c.stream));
    c.fields.push_back(std::move(f));
    return (int)c.fields.size() - 1;
}

void domain_finalize(Ctx& c)
{
    domain_rebuild(c);
    if (c.topology_only) return;
    c.f_source_tmp = field_create(c);
    c.f_target_tmp = field_create(c);
    c.f_correction_tmp = field_create(c);
    c.f_fmm_s = field_create(c);
    c.f_fmm_t = field_create(c);
}

void domain_rebuild(Ctx& c)
{
    HostTree& t = c.tree;
    const std::vector<int> canon = t.canonical();
    c.key_index.clear();
    c.n_leaf_blocks = -1;
    c.n_oct = (int)canon.size();
    for (int i = 0; i < c.n_oct; ++i) t.o[canon[i]].idx = i;
    const int n = c.n_oct;
    c.keys.resize(n);
    c.levels.resize(n);
    c.flags.resize(n);
    c.bbase.resize(3 * (size_t)n);
    c.parent.assign(n, -1);
    c.child.assign(8 * (size_t)n, -1);
    c.level_octs.assign(kMaxLevel + 1, {});
    for (int i = 0; i < n; ++i)
    {
        const HOct& h = t.o[canon[i]];
        c.keys[i] = h.key;
        c.levels[i] = h.level;
        c.flags[i] = (h.leaf ? 1 : 0) | (h.correction ? 2 : 0);
        for (int d = 0; d < 3; ++d) c.bbase[3 * i + d] = h.bbase[d];
        if (h.parent >= 0 && t.o[h.parent].has_data) c.parent[i] = t.o[h.parent].idx;
        for (int k = 0; k < 8; ++k)
            if (h.child[k] >= 0 && t.o[h.child[k]].has_data) c.child[8 * i + k] = t.o[h.child[k]].idx;
        c.level_octs[h.level].push_back(i);
        c.key_index[h.key] = i;
    }
    // neighbour / influence lists on the device
    std::vector<std::pair<u64, int>> sk(n);
    for (int i = 0; i < n; ++i) sk[i] = {c.keys[i], i};
    std::sort(sk.begin(), sk.end());
    std::vector<u64> skeys(n);
    std::vector<int> sidx(n);
    for (int i = 0; i < n; ++i) skeys[i] = sk[i].first, sidx[i] = sk[i].second;
    DevBuf<u64> d_skeys, d_keys;
    DevBuf<int> d_sidx, d_infl, d_ninfl;
    d_skeys.upload(skeys, c.stream);
    d_sidx.upload(sidx, c.stream);
    d_keys.upload(c.keys, c.stream);
    c.d_nbr.alloc(27 * (size_t)n);
    d_infl.alloc(189 * (size_t)n);
    d_ninfl.alloc(n);
    launch_build_lists(c, d_skeys.p, d_sidx.p, n, d_keys.p, n, c.d_nbr.p, d_infl.p, d_ninfl.p);
    c.nbr.resize(27 * (size_t)n);
    c.infl.resize(189 * (size_t)n);
    c.n_infl.resize(n);
    IBLGF_CUDA(cudaMemcpyAsync(c.nbr.data(), c.d_nbr.p, c.nbr.size() * 4, cudaMemcpyDeviceToHost, c.stream));
    IBLGF_CUDA(cudaMemcpyAsync(c.infl.data(), d_infl.p, c.infl.size() * 4, cudaMemcpyDeviceToHost, c.stream));
    IBLGF_CUDA(cudaMemcpyAsync(c.n_infl.data(), d_ninfl.p, n * 4, cudaMemcpyDeviceToHost, c.stream));
    c.d_bbase.upload(c.bbase, c.stream);
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    build_masks(c);
    c.finalized = true;
}

// --------------------------------------------------------------- plans
namespace
{
void upload_tasks(Ctx& c, TpTasks& tt, const std::vector<int>& dst, const std::vector<std::vector<std::pair<int, int>>>& tasks)
{
    std::vector<int> ptr{0}, src, cid, gdst;
    for (size_t g = 0; g < dst.size(); ++g)
    {
        if (tasks[g].empty()) continue;
        gdst.push_back(dst[g]);
        for (auto& t : tasks[g])
        {
            src.push_back(t.first);
            cid.push_back(t.second);
        }
        ptr.push_back((int)src.size());
    }
    tt.n_groups = (int)gdst.size();
    tt.n_tasks = (int)src.size();
    tt.group_ptr.upload(ptr, c.stream);
    tt.group_dst.upload(gdst, c.stream);
    tt.task_src.upload(src, c.stream);
    tt.task_cid.upload(cid, c.stream);
}

// ge < 0: LGF_GL sweep (Fmm::apply full branch); ge >= 0: LGF_GE sweep with
// the integrating-factor table `ge` (neighbour-only branch, fmm.hpp:754-770)
}  // namespace

void host_tasks(HostTasks& ht, const std::vector<int>& dst, const std::vector<std::vector<std::pair<int, int>>>& tasks)
{
    for (size_t g = 0; g < dst.size(); ++g)
    {
        if (tasks[g].empty()) continue;
        ht.dst.push_back(dst[g]);
        for (auto& t : tasks[g])
        {
            ht.src.push_back(t.first);
            ht.cid.push_back(t.second);
        }
        ht.ptr.push_back((int)ht.src.size());
    }
}

void upload_host_tasks(Ctx& c, TpTasks& tt, const HostTasks& ht)
{
    tt.n_groups = (int)ht.dst.size();
    tt.n_tasks = (int)ht.src.size();
    tt.group_ptr.upload(ht.ptr, c.stream);
    tt.group_dst.upload(ht.dst, c.stream);
    tt.task_src.upload(ht.src, c.stream);
    tt.task_cid.upload(ht.cid, c.stream);
}

HostPlan build_host_plan(const Ctx& c, int level, int idx, int ge, bool direct_only)
{
    HostPlan p;
    p.level = level;
    p.mask_idx = idx;
    p.ge = ge;
    const auto& m = c.masks[idx];
    auto S = [&](int o) { return m[2 * o] != 0; };
    auto T = [&](int o) { return m[2 * o + 1] != 0; };
    const bool neighbor_only = ge >= 0;
    // sharded: the targets this rank owns at the sweep level and their
    // ancestors (coarser targets interpolated into them)
    std::vector<char> needed;
    if (!c.owner.empty())
    {
        needed.assign(c.n_oct, 0);
        for (int o : c.level_octs[level])
            for (int a = o; a >= 0 && (a == o ? c.owner[o] == c.rank : !needed[a]); a = c.parent[a]) needed[a] = 1;
    }
    std::vector<int> tgts;
    for (int lv = level; lv >= 0; --lv)
        for (int o : c.level_octs[lv])
        {
            if (S(o)) p.zs.push_back(o);
            if (T(o)) p.zt.push_back(o);
            if (neighbor_only && lv != level) continue;
            if (S(o)) p.srcs.push_back(o);
            if (T(o) && (needed.empty() || needed[o])) tgts.push_back(o);
        }
    for (int o : c.level_octs[level])
    {
        if (S(o)) p.cs.push_back(o);
        if (T(o)) p.at.push_back(o);
    }
    // anterpolation, levels level-1 .. 0
    for (int lv = level - 1; lv >= 0 && !neighbor_only; --lv)
    {
        std::vector<int> dst;
        std::vector<std::vector<std::pair<int, int>>> tasks;
        for (int o : c.level_octs[lv])
        {
            if (!S(o)) continue;
            dst.push_back(o);
            tasks.emplace_back();
            for (int k = 0; k < 8; ++k)
            {
                const int ch = c.child[8 * o + k];
                if (ch >= 0 && S(ch)) tasks.back().push_back({ch, k});
            }
        }
        p.antrp.emplace_back();
        host_tasks(p.antrp.back(), dst, tasks);
    }
    // interpolation, levels 1 .. level-1 (parent level)
    for (int lv = 1; lv < level && !neighbor_only; ++lv)
    {
        std::vector<int> dst;
        std::vector<std::vector<std::pair<int, int>>> tasks;
        for (int o : c.level_octs[lv])
        {
            if (!T(o)) continue;
            for (int k = 0; k < 8; ++k)
            {
                const int ch = c.child[8 * o + k];
                if (ch >= 0 && T(ch) && (needed.empty() || needed[ch]))
                {
                    dst.push_back(ch);
                    tasks.push_back({{o, k}});
                }
            }
        }
        p.intrp.emplace_back();
        host_tasks(p.intrp.back(), dst, tasks);
    }
    // sources and pair list
    std::vector<int> src_slot(c.n_oct, -1);
    for (size_t i = 0; i < p.srcs.size(); ++i) src_slot[p.srcs[i]] = (int)i;
    const int Nb = c.Nb, e = c.cfg.block_extent;
    // reference pair list of every target (fmm.hpp:988-1027, fmm_tt :1167-1195)
    struct TP
    {
        int t;
        std::vector<int> src;
        std::vector<std::array<int, 4>> key;
    };
    std::vector<TP> tp;
    for (int t : tgts)
    {
        const int ld = level - c.levels[t];
        TP x{t, {}, {}};
        auto add_pair = [&](int s, int lvd) {
            x.src.push_back(src_slot[s]);
            x.key.push_back({neighbor_only ? -1 - ge : lvd, c.bbase[3 * t] - c.bbase[3 * s] - (Nb - 1),
                             c.bbase[3 * t + 1] - c.bbase[3 * s + 1] - (Nb - 1),
                             c.bbase[3 * t + 2] - c.bbase[3 * s + 2] - (Nb - 1)});
        };
        if (c.levels[t] == level)
            for (int i = 0; i < 27; ++i)
            {
                const int n = c.nbr[27 * t + i];
                if (n >= 0 && S(n)) add_pair(n, 0);
            }
        for (int i = 0; i < c.n_infl[t] && !neighbor_only; ++i)
        {
            const int n = c.infl[189 * t + i];
            if (n >= 0 && S(n)) add_pair(n, ld);
        }
        if (!x.src.empty()) tp.push_back(std::move(x));
    }
    if (neighbor_only)
        for (auto& x : tp)
        {
            p.ge_tgt.push_back(x.t);
            const size_t b = p.ge_src.size();
            p.ge_src.resize(b + 27, -1);
            for (int s : x.src)
            {
                const int o = p.srcs[s];
                int n = 0, ok = 1;
                for (int a = 0, w = 1; a < 3; ++a, w *= 3)
                {
                    const int d = c.bbase[3 * o + a] - c.bbase[3 * x.t + a];
                    if (d != 0 && d != e && d != -e) ok = 0;
                    n += (d / e + 1) * w;
                }
                if (!ok || p.ge_src[b + n] != -1) throw Error(IBLGF_EINTERNAL, "neighbour-only source is not an adjacent block");
                p.ge_src[b + n] = o;
            }
        }
    if (neighbor_only && direct_only)
    {
        // the direct sweep needs the targets and their neighbour sources only
        p.tgt_list = p.ge_tgt;
        return p;
    }
    // sibling groups: a target joins its parent's group when the structured
    // candidate set (children of the parent's 27 neighbours; non-adjacent ones
    // only below the sweep level) reproduces its pair list exactly
    struct Grp
    {
        u64 pkey;
        int ld;
        std::array<int, 8> tgt;
        std::array<int, 216> cand;  // source slot or -1
        std::array<bool, 216> used;
    };
    std::map<std::pair<int, u64>, int> gidx;
    std::vector<Grp> groups;
    std::vector<char> in_group(tp.size(), 0);
    auto adjacent = [](int cc, int k) {
        const int n = k / 8, cp = k % 8;
        const int ux = (cc & 1) - (cp & 1) - 2 * (n % 3 - 1);
        const int uy = ((cc >> 1) & 1) - ((cp >> 1) & 1) - 2 * ((n / 3) % 3 - 1);
        const int uz = ((cc >> 2) & 1) - ((cp >> 2) & 1) - 2 * (n / 9 - 1);
        return std::abs(ux) <= 1 && std::abs(uy) <= 1 && std::abs(uz) <= 1;
    };
    for (size_t i = 0; i < tp.size(); ++i)
    {
        const int t = tp[i].t;
        if (c.levels[t] == 0) continue;
        const int ld = level - c.levels[t];
        const u64 pk = key_parent(c.keys[t]);
        const int cc = key_child_number(c.keys[t], c.levels[t]);
        std::array<int, 216> cand;
        int k = 0;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx)
                {
                    const u64 pn = key_neighbor(pk, dx, dy, dz);
                    for (int cp = 0; cp < 8; ++cp, ++k)
                    {
                        auto it = c.key_index.find(key_child(pn, cp));
                        const int o = it == c.key_index.end() ? -1 : it->second;
                        cand[k] = (o >= 0 && S(o)) ? src_slot[o] : -1;
                    }
                }
        const int mode = neighbor_only ? 2 : (ld == 0 ? 0 : 1);
        auto valid = [&](int kk) {
            return mode == 0 || (mode == 1 && !adjacent(cc, kk)) || (mode == 2 && adjacent(cc, kk));
        };
        std::vector<int> mine;
        for (int kk = 0; kk < 216; ++kk)
            if (cand[kk] >= 0 && valid(kk)) mine.push_back(cand[kk]);
        std::vector<int> ref = tp[i].src;
        std::sort(mine.begin(), mine.end());
        std::sort(ref.begin(), ref.end());
        if (mine != ref) continue;
        auto key = std::make_pair(c.levels[t], pk);
        auto it = gidx.find(key);
        int g;
        if (it == gidx.end())
        {
            g = (int)groups.size();
            gidx.emplace(key, g);
            Grp gr;
            gr.pkey = pk;
            gr.ld = ld;
            gr.tgt.fill(-1);
            gr.cand = cand;
            gr.used.fill(false);
            groups.push_back(gr);
        }
        else
            g = it->second;
        groups[g].tgt[cc] = (int)i;  // temporary: index into tp
        for (int kk = 0; kk < 216; ++kk)
            if (cand[kk] >= 0 && valid(kk)) groups[g].used[kk] = true;
        in_group[i] = 1;
    }
    // target slots: pair-list targets first, then group targets in group order
    std::vector<int> slot_of_tp(tp.size(), -1);
    for (size_t i = 0; i < tp.size(); ++i)
    {
        if (in_group[i]) continue;
        slot_of_tp[i] = (int)p.tgt_list.size();
        p.tgt_list.push_back(tp[i].t);
        p.psrc.insert(p.psrc.end(), tp[i].src.begin(), tp[i].src.end());
        p.pkey.insert(p.pkey.end(), tp[i].key.begin(), tp[i].key.end());
        p.ptr.push_back((int)p.psrc.size());
    }
    p.n_csr_tgt = (int)p.tgt_list.size();
    // groups ordered by (sweep level distance, parent key): spatially coherent tiles
    std::vector<int> gorder(groups.size());
    for (size_t g = 0; g < groups.size(); ++g) gorder[g] = (int)g;
    std::sort(gorder.begin(), gorder.end(), [&](int a, int b) {
        return groups[a].ld != groups[b].ld ? groups[a].ld < groups[b].ld : groups[a].pkey < groups[b].pkey;
    });
    for (int g : gorder)
        for (int cc = 0; cc < 8; ++cc)
        {
            const int i = groups[g].tgt[cc];
            if (i < 0) continue;
            slot_of_tp[i] = (int)p.tgt_list.size();
            p.tgt_list.push_back(tp[i].t);
        }
    // per-ld spectrum slot tables over the 343 offsets
    std::map<int, int> tab_of_ld;
    for (auto& gr : groups)
    {
        if (tab_of_ld.count(gr.ld)) continue;
        tab_of_ld[gr.ld] = (int)tab_of_ld.size();
        for (int u = 0; u < 343; ++u)
        {
            const int ux = u % 7 - 3, uy = (u / 7) % 7 - 3, uz = u / 49 - 3;
            p.tab_keys.push_back({neighbor_only ? -1 - ge : gr.ld, ux * e - (Nb - 1), uy * e - (Nb - 1),
                                  uz * e - (Nb - 1)});
        }
    }
    // tiles: consecutive groups of one level distance while the union of their
    // sources fits the staging budget
    // a tile: up to 32 sibling groups (16 rows x 2 per row of the MAC CTA) whose
    // union of candidate sources fits the 64-byte-row staging budget
    const int kScap = 1024, kGcap = kGroupTileCap;
    std::vector<int>& tgptr = p.tgptr;
    std::vector<int>& tsptr = p.tsptr;
    std::vector<int>& tsrc = p.tsrc;
    std::vector<int>& ttab = p.ttab;
    std::vector<int>& tcoarse = p.tcoarse;
    std::vector<int>& gtgt = p.gtgt;
    std::vector<unsigned short>& gsrc = p.gsrc;
    std::vector<unsigned>& gpm = p.gpm;
    std::map<int, int> local;
    int cur_ld = -1, ngrp = 0, max_src = 0;
    auto close_tile = [&]() {
        if (!ngrp) return;
        tgptr.push_back((int)gtgt.size() / 8);
        tsptr.push_back((int)tsrc.size());
        ttab.push_back(tab_of_ld[cur_ld]);
        tcoarse.push_back(neighbor_only ? 2 : (cur_ld > 0 ? 1 : 0));
        max_src = std::max(max_src, (int)local.size());
        local.clear();
        ngrp = 0;
    };
    for (int g : gorder)
    {
        const Grp& gr = groups[g];
        int extra = 0;
        for (int kk = 0; kk < 216; ++kk)
            if (gr.used[kk] && !local.count(gr.cand[kk])) ++extra;
        if (ngrp && (gr.ld != cur_ld || ngrp >= kGcap || (int)local.size() + extra > kScap)) close_tile();
        cur_ld = gr.ld;
        for (int kk = 0; kk < 216; ++kk)
        {
            if (!gr.used[kk])
            {
                gsrc.push_back(0xFFFF);
                continue;
            }
            auto it = local.find(gr.cand[kk]);
            int j;
            if (it == local.end())
            {
                j = (int)local.size();
                local.emplace(gr.cand[kk], j);
                tsrc.push_back(gr.cand[kk]);
            }
            else
                j = it->second;
            gsrc.push_back((unsigned short)j);
        }
        for (int cc = 0; cc < 8; ++cc) gtgt.push_back(gr.tgt[cc] >= 0 ? slot_of_tp[gr.tgt[cc]] : -1);
        unsigned pm = 0;
        for (int kk = 0; kk < 216; ++kk)
            if (gr.used[kk]) pm |= 1u << (kk / 8);
        gpm.push_back(pm);
        // the kernel runs all 64 (c, c') products of a present parent, or
        // only the adjacent ones when the plan is neighbour-only
        for (int n = 0; n < 27; ++n)
            if (pm >> n & 1u)
            {
                int cnt = 1;
                for (int a = 0; a < 3; ++a)
                    cnt *= (neighbor_only && (n / (a == 0 ? 1 : (a == 1 ? 3 : 9))) % 3 != 1) ? 1 : 4;
                p.n_exec += cnt;
            }
        ++ngrp;
    }
    close_tile();
    p.n_groups = (int)groups.size();
    p.max_tile_src = max_src;
    for (auto& x : tp) p.all_keys.insert(p.all_keys.end(), x.key.begin(), x.key.end());
    for (auto& x : tp) p.n_pairs += (long long)x.src.size();
    p.n_exec += (long long)p.psrc.size();  // pair-list targets
    {
        std::vector<std::array<int, 4>> u;
        for (auto& x : tp) u.insert(u.end(), x.key.begin(), x.key.end());
        std::sort(u.begin(), u.end());
        p.n_spec_unique = (int)(std::unique(u.begin(), u.end()) - u.begin());
    }
    return p;
}

std::unique_ptr<FmmPlan> upload_plan(Ctx& c, const HostPlan& h)
{
    auto plan = std::make_unique<FmmPlan>();
    FmmPlan& p = *plan;
    p.level = h.level;
    p.mask_idx = h.mask_idx;
    p.zero_s.upload(h.zs, c.stream);
    p.zero_t.upload(h.zt, c.stream);
    p.copy_s.upload(h.cs, c.stream);
    p.add_t.upload(h.at, c.stream);
    for (auto& t : h.antrp)
    {
        p.antrp.emplace_back();
        upload_host_tasks(c, p.antrp.back(), t);
    }
    for (auto& t : h.intrp)
    {
        p.intrp.emplace_back();
        upload_host_tasks(c, p.intrp.back(), t);
    }
    p.n_src = (int)h.srcs.size();
    p.src_oct.upload(h.srcs, c.stream);
    // LGF spectrum slots: every pair's key gets a slot (new ones are computed
    // below); the group tables reference registered keys only (-1: zero row)
    std::vector<std::array<int, 5>> new_slots;
    auto slot_of = [&](const std::array<int, 4>& k) {
        auto it = c.spec_slot.find(k);
        if (it != c.spec_slot.end()) return it->second;
        const int slot = (int)c.spec_slot.size();
        c.spec_slot.emplace(k, slot);
        new_slots.push_back({slot, k[0], k[1], k[2], k[3]});
        return slot;
    };
    for (auto& k : h.all_keys) slot_of(k);
    // the block-Toeplitz MAC reads all 343 offsets of a table (absent
    // sources multiply zero rows): every offset gets its spectrum
    const bool toeplitz = !h.ttab.empty() && h.ge < 0 && c.cfg.precision == IBLGF_FP32;
    if (toeplitz)
        for (auto& k : h.tab_keys) slot_of(k);
    std::vector<int> pspec(h.pkey.size());
    for (size_t i = 0; i < h.pkey.size(); ++i) pspec[i] = slot_of(h.pkey[i]);
    std::vector<int> spec_u(h.tab_keys.size());
    for (size_t i = 0; i < h.tab_keys.size(); ++i)
    {
        auto it = c.spec_slot.find(h.tab_keys[i]);
        spec_u[i] = it == c.spec_slot.end() ? -1 : it->second;
    }
    p.n_csr_tgt = h.n_csr_tgt;
    p.n_groups = h.n_groups;
    p.n_ge = (int)h.ge_tgt.size();
    if (p.n_ge)
    {
        p.ge_tgt.upload(h.ge_tgt, c.stream);
        p.ge_src.upload(h.ge_src, c.stream);
    }
    p.n_tiles = (int)h.ttab.size();
    p.max_tile_src = h.max_tile_src;
    p.tile_gptr.upload(h.tgptr, c.stream);
    {
        // candidate source rows per tile: group g's candidate kk reads row
        // tsrc[tsptr[t] + gsrc[g][kk]], absent ones (and unused group slots)
        // the zero row n_src
        // padded so that the block-Toeplitz MAC's copy of a tile's last part
        // (3 parts of kToeplitzPart rows) stays inside the buffer
        const size_t pad = (size_t)(3 * kToeplitzPart - kGroupTileCap) * 216;
        std::vector<int> jr((size_t)p.n_tiles * kGroupTileCap * 216 + pad, p.n_src);
        for (int t = 0; t < p.n_tiles; ++t)
            for (int g = h.tgptr[t]; g < h.tgptr[t + 1]; ++g)
                for (int kk = 0; kk < 216; ++kk)
                {
                    const unsigned short j = h.gsrc[(size_t)g * 216 + kk];
                    if (j != 0xFFFF)
                        jr[((size_t)t * kGroupTileCap + (g - h.tgptr[t])) * 216 + kk] = h.tsrc[h.tsptr[t] + j];
                }
        p.tile_jr.upload(jr, c.stream);
        // the same rows per group for the tensor-core MAC, whose tiles span
        // up to 128 consecutive groups
        std::vector<int> gjr((size_t)std::max(h.n_groups, 1) * 216, p.n_src);
        for (int t = 0; t < p.n_tiles; ++t)
            for (int g = h.tgptr[t]; g < h.tgptr[t + 1]; ++g)
                std::copy_n(jr.begin() + ((size_t)t * kGroupTileCap + (g - h.tgptr[t])) * 216, 216,
                            gjr.begin() + (size_t)g * 216);
        if (p.n_tiles) p.grp_jr.upload(gjr, c.stream);
        std::vector<int> tg, tt, tm;
        std::vector<unsigned> tp;
        build_tc_tiles(h.tgptr, h.ttab, h.tcoarse, h.gpm, tg, tt, tm, tp);
        p.n_tc = (int)tt.size();
        if (p.n_tc)
        {
            p.tc_gptr.upload(tg, c.stream);
            p.tc_tab.upload(tt, c.stream);
            p.tc_mode.upload(tm, c.stream);
            p.tc_pm.upload(tp, c.stream);
        }
    }
    p.tile_tab.upload(h.ttab, c.stream);
    p.tile_coarse.upload(h.tcoarse, c.stream);
    p.spec_u.upload(spec_u, c.stream);
    p.grp_pm.upload(h.gpm, c.stream);
    p.grp_tgt.upload(h.gtgt, c.stream);
    p.n_exec = h.n_exec;
    p.adj_only = !h.tcoarse.empty();
    for (int m : h.tcoarse) p.adj_only = p.adj_only && m == 2;
    // MAC work per frequency: 8 flops per complex multiply-add of the direct
    // kernels; the block-Toeplitz kernel per (group, present parent) 27
    // complex multiply-adds and 19 complex additions, and per group the 38
    // additions of the final combination
    p.mac_flops = (long long)h.psrc.size() * 8;
    if (p.adj_only || !toeplitz)
        p.mac_flops += (h.n_exec - (long long)h.psrc.size()) * 8;
    else
        for (unsigned pm : h.gpm) p.mac_flops += (long long)__builtin_popcount(pm) * (27 * 8 + 19 * 2) + 38 * 2;
    p.n_tgt = (int)h.tgt_list.size();
    p.n_pairs = h.n_pairs;
    p.n_spec_unique = h.n_spec_unique;
    p.tgt_oct.upload(h.tgt_list, c.stream);
    p.pair_ptr.upload(h.ptr, c.stream);
    p.pair_src.upload(h.psrc, c.stream);
    p.pair_spec.upload(pspec, c.stream);
    // grow the spectra cache and fill the new slots
    if (!new_slots.empty())
    {
        const int need = (int)c.spec_slot.size();
        if (need > c.spec_cap)
        {
            const int cap = std::max(need, c.spec_cap * 2);
            DevBuf<char> nb;
            nb.alloc((size_t)cap * c.NC * c.cplx_bytes());
            if (c.spec_used)
                IBLGF_CUDA(cudaMemcpyAsync(nb.p, c.d_spec.p, (size_t)c.spec_used * c.NC * c.cplx_bytes(),
                                           cudaMemcpyDeviceToDevice, c.stream));
            IBLGF_CUDA(cudaStreamSynchronize(c.stream));
            c.d_spec = std::move(nb);
            c.spec_cap = cap;
        }
        launch_spectra(c, new_slots);
        c.spec_used = need;
    }
    if (toeplitz && !p.adj_only)
    {
        std::vector<int> tcombo(h.ttab.size());
        std::vector<int> of_tab(h.tab_keys.size() / 343, -1);
        for (size_t t = 0; t < of_tab.size(); ++t)
        {
            const std::vector<int> slots(spec_u.begin() + 343 * t, spec_u.begin() + 343 * (t + 1));
            of_tab[t] = combo_table(c, h.tab_keys[343 * t][0], slots);
        }
        for (size_t i = 0; i < h.ttab.size(); ++i) tcombo[i] = of_tab[h.ttab[i]];
        p.tile_combo.upload(tcombo, c.stream);
        std::vector<int> parts;
        for (size_t t = 0; t + 1 < h.tgptr.size(); ++t)
            for (int q = 0; q * kToeplitzPart < h.tgptr[t + 1] - h.tgptr[t]; ++q) parts.push_back((int)(t << 2) | q);
        p.n_parts = (int)parts.size();
        p.tile_parts.upload(parts, c.stream);
    }
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    return plan;
}

namespace
{
FmmPlan& get_plan(Ctx& c, int level, int idx, int ge)
{
    // neighbour-only plans for the direct sweep are built without the
    // transform path's pair lists, groups and spectra (keyed apart)
    const bool direct = ge >= 0 && c.ge_direct_enabled && ge_direct_ok(c, ge);
    auto key = std::make_tuple(idx, level, ge < 0 ? -1 : 2 * ge + (direct ? 1 : 0));
    auto it = c.plans.find(key);
    if (it != c.plans.end()) return *it->second;
    const auto t0 = std::chrono::steady_clock::now();
    HostPlan h = build_host_plan(c, level, idx, ge, direct);
    const auto t1 = std::chrono::steady_clock::now();
    auto plan = upload_plan(c, h);
    if (c.trace)
    {
        const auto t2 = std::chrono::steady_clock::now();
        std::fprintf(stderr, "iblgf plan level %d mask %d ge %d%s: %zu targets, %lld pairs; build %.2f ms, upload %.2f ms\n",
                     level, idx, ge, direct ? " (direct)" : "", h.tgt_list.size(), h.n_pairs,
                     std::chrono::duration<double, std::milli>(t1 - t0).count(),
                     std::chrono::duration<double, std::milli>(t2 - t1).count());
    }
    auto& ref = *plan;
    c.plans.emplace(key, std::move(plan));
    return ref;
}

}  // namespace

// Rebuilds the plans of the given keys (the sweeps that existed before an
// adaptation) for the current octree: the host plans are built on parallel
// host threads (build_host_plan only reads the context), then uploaded in
// key order on the context stream. Keys whose level or mask no longer exists
// are skipped; the first sweep that needs one builds it as before.
void prebuild_plans(Ctx& c, const std::vector<std::tuple<int, int, int>>& keys)
{
    if (!c.owner.empty()) return;
    std::vector<std::tuple<int, int, int>> todo;
    for (const auto& k : keys)
    {
        const int idx = std::get<0>(k), level = std::get<1>(k);
        if (idx < 0 || idx >= (int)c.masks.size() || level < c.tree.base_level || level >= c.tree.depth) continue;
        if (!c.plans.count(k)) todo.push_back(k);
    }
    if (todo.empty()) return;
    std::vector<HostPlan> hp(todo.size());
    std::vector<std::string> err(todo.size());
    std::atomic<size_t> next{0};
    auto work = [&]() {
        for (size_t i = next++; i < todo.size(); i = next++)
        {
            const int idx = std::get<0>(todo[i]), level = std::get<1>(todo[i]), gk = std::get<2>(todo[i]);
            try
            {
                hp[i] = build_host_plan(c, level, idx, gk < 0 ? -1 : gk / 2, gk >= 0 && (gk & 1));
            }
            catch (const std::exception& e)
            {
                err[i] = e.what();
            }
        }
    };
    const unsigned hw = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned k = 1; k < std::min<unsigned>(hw, (unsigned)todo.size()); ++k) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
    for (size_t i = 0; i < todo.size(); ++i)
    {
        if (!err[i].empty()) continue;  // rebuilt on first use instead
        c.plans.emplace(todo[i], upload_plan(c, hp[i]));
    }
}

namespace
{
void ensure_bytes(DevBuf<char>& b, size_t bytes)
{
    if (b.n < bytes) b.alloc(bytes);
}

struct Timer
{
    // phase events recorded on the context stream; read back (and summed) by
    // iblgf_profile_read, so profiling adds no host synchronisation
    Ctx& c;
    std::array<cudaEvent_t, 5> ev{};
    bool on;
    explicit Timer(Ctx& cc)
    : c(cc)
    , on(cc.profile)
    {
        if (on)
            for (auto& e : ev) IBLGF_CUDA(cudaEventCreate(&e));
    }
    void mark(int i)
    {
        if (on) IBLGF_CUDA(cudaEventRecord(ev[i], c.stream));
    }
    ~Timer()
    {
        if (on) c.prof_events.push_back(ev);
    }
};
}  // namespace

// Domain::construct_basemesh_blocks (domain.hpp:405-488): blocks given as
// boxes of base cells, each split into block_extent^3 base blocks
void add_blocks(Ctx& c, int n, const int* base, const int* extent)
{
    if (n < 0 || (n && (!base || !extent))) throw Error(IBLGF_EINVAL, "bad block arguments");
    const int e = c.cfg.block_extent;
    std::vector<std::array<int, 3>> nb;
    for (int b = 0; b < n; ++b)
    {
        for (int d = 0; d < 3; ++d)
        {
            if (extent[3 * b + d] <= 0 || extent[3 * b + d] % e)
                throw Error(IBLGF_EINVAL, "Domain: Extent of blocks are not evenly divisible");
            if (std::abs(base[3 * b + d]) % e)
                throw Error(IBLGF_EINVAL, "Domain: Base of blocks are not evenly divisible");
        }
        for (int k = 0; k < extent[3 * b + 2] / e; ++k)
            for (int j = 0; j < extent[3 * b + 1] / e; ++j)
                for (int i = 0; i < extent[3 * b] / e; ++i)
                    nb.push_back({base[3 * b] / e + i, base[3 * b + 1] / e + j, base[3 * b + 2] / e + k});
    }
    c.tree.add_base_blocks(nb);
    c.has_blocks = true;
}

void need_single(const Ctx& c)
{
    if (c.batch) throw Error(IBLGF_EINVAL, "the context holds a batch of problems (use the iblgf_batch_* calls)");
}

void fmm_apply(Ctx& c, int src, int tgt, int level, bool nlas, double add_with_scale, int fmm_type, int ge)
{
    need_single(c);
    if (!c.finalized) throw Error(IBLGF_EINVAL, "domain not finalized");
    if (level < c.tree.base_level || level >= c.tree.depth) throw Error(IBLGF_EINVAL, "level out of range");
    const int rl = level - c.tree.base_level;
    const int idx = fmm_type == IBLGF_AMR2AMR ? mask_idx_gen(IBLGF_AMR2AMR, rl, nlas ? 1 : 0)
                                               : mask_idx_gen(fmm_type, rl, 0);
    FmmPlan& p = get_plan(c, level, idx, ge);
    run_sweep(c, p, src, tgt, c.cfg.dx_base / std::pow(2.0, rl), add_with_scale, ge);
}

void run_sweep(Ctx& c, FmmPlan& p, int src, int tgt, double dx_level, double add_with_scale, int ge)
{
    c.stats[0] += 1;
    c.stats[1] += p.n_src;
    c.stats[2] += p.n_tgt;
    c.stats[3] += p.n_pairs;
    c.stats[4] += p.n_spec_unique;
    for (auto& t : p.antrp) c.stats[5] += t.n_tasks;
    for (auto& t : p.intrp) c.stats[6] += t.n_tasks;
    c.stats[7] += p.n_tgt - p.n_csr_tgt;
    c.stats[9] += p.mac_flops;
    c.stats[8] += p.n_exec;
    double* fs = c.field(c.f_fmm_s);
    double* ft = c.field(c.f_fmm_t);
    Timer tm(c);
    tm.mark(0);
    launch_zero_blocks(c, fs, p.zero_s.p, (int)p.zero_s.n);
    launch_zero_blocks(c, ft, p.zero_t.p, (int)p.zero_t.n);
    launch_copy_interior(c, c.field(src), fs, p.copy_s.p, (int)p.copy_s.n);
    // the FMM's Lagrange anterpolation of the sources (fmm_nli.hpp) runs its
    // passes in FP32 on the FP32 path (the coarse sources feed FP32
    // transforms); the interpolation of the targets stays FP64
    const bool fp32 = c.cfg.precision == IBLGF_FP32;
    for (auto& t : p.antrp) launch_tp(c, t, fs, fs, 0, 0, fp32);
    tm.mark(1);
    const size_t cb = c.cplx_bytes();
    // integrating-factor sweeps whose kernel is negligible beyond 8 cells:
    // direct separable sums instead of transforms (same result to FP64 rounding)
    const bool direct = ge >= 0 && c.ge_direct_enabled && p.n_ge && ge_direct_ok(c, ge);
    if (!p.empty() && !direct)
    {
        // the source spectra and one zero row after them (absent MAC candidates read it)
        ensure_bytes(c.d_src_spec, (size_t)(p.n_src + 1) * c.NC * cb);
        launch_fill_zero(c, reinterpret_cast<double*>(c.d_src_spec.p + (size_t)p.n_src * c.NC * cb),
                         c.NC * cb / sizeof(double));
        ensure_bytes(c.d_acc, (size_t)p.n_tgt * c.NC * cb);
        launch_forward_sources(c, fs, p.src_oct.p, p.n_src, c.d_src_spec.p);
    }
    tm.mark(2);
    if (!p.empty() && !direct) launch_mac(c, p, c.d_src_spec.p, c.d_acc.p);
    tm.mark(3);
    if (!p.empty() && direct) launch_ge_direct(c, p, fs, ft, ge, 1.0);
    else if (!p.empty())
    {
        // compute_influence_field (fmm.hpp:1021-1026): dx^2 for LGF_GL, 1 for LGF_GE
        const double scale = (ge >= 0 ? 1.0 : dx_level * dx_level) / ((double)c.P * c.P * c.P);
        launch_inverse_add(c, p, c.d_acc.p, ft, scale);
    }
    for (auto& t : p.intrp) launch_tp(c, t, ft, ft, 0, 1);
    if (!c.owner.empty() && p.add_t.n)
    {
        // sharded: sum the level targets' results over the ranks
        const size_t count = p.add_t.n * c.block_elems();
        if (c.exchange_buf.n < count) c.exchange_buf.alloc(count, c.cfg.device, c.stream);
        launch_blocks_gather(c, ft, c.exchange_buf.p, p.add_t.p, (int)p.add_t.n);
        if (!c.exchange_fn) throw Error(IBLGF_EINVAL, "sharded sweep without an exchange callback");
        if (c.exchange_fn(c.exchange_user, c.exchange_buf.p, count, (void*)c.stream) != 0)
            throw Error(IBLGF_EINTERNAL, "the exchange callback failed");
        launch_blocks_scatter(c, c.exchange_buf.p, ft, p.add_t.p, (int)p.add_t.n);
    }
    launch_axpy_blocks(c, ft, c.field(tgt), p.add_t.p, (int)p.add_t.n, add_with_scale, false);
    tm.mark(4);
}

// --------------------------------------------------------------- Poisson
PoissonLists& poisson_lists(Ctx& c)
{
    if (auto* have = c.ext_get<PoissonLists>(Ctx::kExtPLists)) return *have;
    auto pl = std::make_unique<PoissonLists>();
    std::vector<int> all, leaves;
    for (int i = 0; i < c.n_oct; ++i)
    {
        all.push_back(i);
        if (c.flags[i] & 1) leaves.push_back(i);
    }
    pl->all.upload(all, c.stream);
    pl->leaves.upload(leaves, c.stream);
    const int L = kMaxLevel + 1;
    pl->level_all.resize(L);
    pl->level_leaves.resize(L);
    pl->coarsify.resize(L);
    pl->cc_intrp.resize(L);
    pl->corr_intrp.resize(L);
    pl->children.resize(L);
    for (int l = 0; l < (int)c.level_octs.size(); ++l)
    {
        std::vector<int> la, ll, ch;
        std::vector<int> cdst, idst, kdst;
        std::vector<std::vector<std::pair<int, int>>> ctasks, itasks, ktasks;
        for (int o : c.level_octs[l])
        {
            la.push_back(o);
            if (c.flags[o] & 1) ll.push_back(o);
            cdst.push_back(o);
            ctasks.emplace_back();
            for (int k = 0; k < 8; ++k)
            {
                const int x = c.child[8 * o + k];
                if (x < 0) continue;
                ctasks.back().push_back({x, k});
                idst.push_back(x);
                itasks.push_back({{o, k}});
                ch.push_back(x);
                if (c.flags[x] & 2)
                {
                    kdst.push_back(x);
                    ktasks.push_back({{o, k}});
                }
            }
        }
        pl->level_all[l].upload(la, c.stream);
        pl->level_leaves[l].upload(ll, c.stream);
        pl->children[l].upload(ch, c.stream);
        upload_tasks(c, pl->coarsify[l], cdst, ctasks);
        upload_tasks(c, pl->cc_intrp[l], idst, itasks);
        upload_tasks(c, pl->corr_intrp[l], kdst, ktasks);
    }
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    auto& ref = *pl;
    c.ext[Ctx::kExtPLists] = std::shared_ptr<PoissonLists>(std::move(pl));
    return ref;
}

// per level (and "all levels" at index kMaxLevel+1): block list and dx per block
OpLists& op_lists(Ctx& c)
{
    if (auto* have = c.ext_get<OpLists>(Ctx::kExtOpLists)) return *have;
    auto ol = std::make_unique<OpLists>();
    const int L = kMaxLevel + 2;
    ol->list.resize(L);
    ol->dx.resize(L);
    std::vector<int> all;
    std::vector<double> alldx;
    for (int l = 0; l <= kMaxLevel; ++l)
    {
        std::vector<double> dx;
        const double d = c.cfg.dx_base / std::pow(2.0, l - c.tree.base_level);
        for (int o : c.level_octs[l])
        {
            dx.push_back(d);
            all.push_back(o);
            alldx.push_back(d);
        }
        ol->list[l].upload(c.level_octs[l], c.stream);
        ol->dx[l].upload(dx, c.stream);
    }
    ol->list[L - 1].upload(all, c.stream);
    ol->dx[L - 1].upload(alldx, c.stream);
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    auto& ref = *ol;
    c.ext[Ctx::kExtOpLists] = std::shared_ptr<OpLists>(std::move(ol));
    return ref;
}

void buffer_exchange(Ctx& c, int field, int level)
{
    need_single(c);
    if (level < 0 || level > kMaxLevel) throw Error(IBLGF_EINVAL, "level out of range");
    OpLists& ol = op_lists(c);
    launch_halo(c, c.field(field), ol.list[level].p, (int)ol.list[level].n);
}

void apply_op(Ctx& c, int op, const int* in, int n_in, const int* out, int n_out, int level, double scale)
{
    need_single(c);
    static const int need_in[6] = {1, 1, 3, 3, 3, 6}, need_out[6] = {1, 3, 1, 3, 3, 3};
    if (op < 0 || op > 5) throw Error(IBLGF_EINVAL, "unknown operator");
    if (n_in != need_in[op] || n_out != need_out[op]) throw Error(IBLGF_EINVAL, "wrong number of component fields");
    if (level > kMaxLevel) throw Error(IBLGF_EINVAL, "level out of range");
    OpLists& ol = op_lists(c);
    const int li = level < 0 ? kMaxLevel + 1 : level;
    const double* pin[6] = {};
    double* pout[3] = {};
    for (int i = 0; i < n_in; ++i) pin[i] = c.field(in[i]);
    for (int i = 0; i < n_out; ++i)
    {
        pout[i] = c.field(out[i]);
        for (int j = 0; j < n_in; ++j)
            if (out[i] == in[j]) throw Error(IBLGF_EINVAL, "operator output aliases an input");
    }
    launch_op(c, op, pin, n_in, pout, n_out, ol.list[li].p, ol.dx[li].p, (int)ol.list[li].n, scale);
}

// The block operators on a list of octants (Operator::laplace ... applied to
// it->data() with the octant's dx_level, operators.hpp:1386-1513, 2416-2531)
void apply_op_octants(Ctx& c, int op, const int* in, int n_in, const int* out, int n_out, const int* octants, int n,
                      double scale)
{
    need_single(c);
    static const int need_in[6] = {1, 1, 3, 3, 3, 6}, need_out[6] = {1, 3, 1, 3, 3, 3};
    if (op < 0 || op > 5) throw Error(IBLGF_EINVAL, "unknown operator");
    if (n_in != need_in[op] || n_out != need_out[op]) throw Error(IBLGF_EINVAL, "wrong number of component fields");
    if (n <= 0) return;
    std::vector<int> list(octants, octants + n);
    std::vector<double> dx(n);
    for (int i = 0; i < n; ++i)
    {
        if (list[i] < 0 || list[i] >= c.n_oct) throw Error(IBLGF_EINVAL, "octant out of range");
        dx[i] = c.cfg.dx_base / std::pow(2.0, c.levels[list[i]] - c.tree.base_level);
    }
    const double* pin[6] = {};
    double* pout[3] = {};
    for (int i = 0; i < n_in; ++i) pin[i] = c.field(in[i]);
    for (int i = 0; i < n_out; ++i)
    {
        pout[i] = c.field(out[i]);
        for (int j = 0; j < n_in; ++j)
            if (out[i] == in[j]) throw Error(IBLGF_EINVAL, "operator output aliases an input");
    }
    DevBuf<int> d_list;
    DevBuf<double> d_dx;
    d_list.upload(list, c.stream);
    d_dx.upload(dx, c.stream);
    launch_op(c, op, pin, n_in, pout, n_out, d_list.p, d_dx.p, n, scale);
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));  // the lists are freed on return
}

// e^{-2 alpha} I_n(2 alpha), n = 0..stride-1, by Miller's backward recurrence
// normalised with e^x = I_0 + 2 sum I_k (A&S 9.6.26, 9.6.37)
int ge_table(Ctx& c, double alpha)
{
    auto it = c.ge_index.find(alpha);
    if (it != c.ge_index.end()) return it->second;
    if (!(alpha >= 0.0)) throw Error(IBLGF_EINVAL, "integrating-factor alpha must be non-negative");
    c.ge_stride = 4 * c.Nb + 9;
    const int nmax = c.ge_stride - 1;
    const double x = 2.0 * alpha;
    std::vector<double> f(c.ge_stride, 0.0);
    if (alpha == 0.0)
    {
        // e^0 I_n(0) = [n == 0]: the identity (the recurrence divides by x)
        f[0] = 1.0;
        const int idx = (int)c.ge_index.size();
        c.ge_index.emplace(alpha, idx);
        c.ge_host.insert(c.ge_host.end(), f.begin(), f.end());
        c.d_ge.upload(c.ge_host, c.stream);
        IBLGF_CUDA(cudaStreamSynchronize(c.stream));
        return idx;
    }
    const int m = nmax + 30 + (int)std::ceil(std::sqrt(90.0 * x));
    double a = 0.0, b = 1e-280, sum = 0.0;
    for (int k = m; k >= 1; --k)
    {
        const double cc = a + (2.0 * k / x) * b;
        sum += b;
        if (k <= nmax) f[k] = b;
        a = b;
        b = cc;
        if (std::fabs(b) > 1e250)
        {
            a *= 1e-250;
            b *= 1e-250;
            sum *= 1e-250;
            for (int n = k; n <= nmax; ++n) f[n] *= 1e-250;
        }
    }
    f[0] = b;
    const double norm = b + 2.0 * sum;
    for (auto& v : f) v /= norm;
    const int idx = (int)c.ge_index.size();
    c.ge_index.emplace(alpha, idx);
    c.ge_host.insert(c.ge_host.end(), f.begin(), f.end());
    c.d_ge.upload(c.ge_host, c.stream);
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    return idx;
}

// PoissonSolver::apply_lgf_IF / apply_if (poisson.hpp:428-494), AMR2AMR
void apply_if(Ctx& c, int src, int tgt, double alpha_base, int fmm_type, const int* rp)
{
    need_single(c);
    static const int cell[3] = {1, 1, 1};
    if (!rp) rp = cell;
    // cell-centred transfer matrices per axis: relative position 1 -> [4,5]
    // coarsify / [2,3] interpolate, relative position 0 -> [8,9] / [6,7]
    const int coarse_m[3] = {rp[0] ? 4 : 8, rp[1] ? 4 : 8, rp[2] ? 4 : 8};
    const int intrp_m[3] = {rp[0] ? 2 : 6, rp[1] ? 2 : 6, rp[2] ? 2 : 6};
    if (!c.finalized) throw Error(IBLGF_EINVAL, "domain not finalized");
    if (fmm_type != IBLGF_AMR2AMR && fmm_type != IBLGF_IB2xIB)
        throw Error(IBLGF_EINVAL, "apply_if supports AMR2AMR and IB2xIB");
    PoissonLists& pl = poisson_lists(c);
    OpLists& ol = op_lists(c);
    double* st = c.field(c.f_source_tmp);
    double* tt = c.field(c.f_target_tmp);
    const size_t bytes = c.field_elems() * sizeof(double);
    launch_fill_zero(c, st, bytes / sizeof(double));
    launch_fill_zero(c, tt, bytes / sizeof(double));
    const int bl = c.tree.base_level, depth = c.tree.depth;
    if (fmm_type == IBLGF_IB2xIB)
    {
        // poisson.hpp:447-448, 465-494: finest level only, interior copy, the
        // non-leaf-as-source sweep with the IB2xIB mask, level copied out
        const int l = depth - 1;
        launch_copy_interior(c, c.field(src), st, pl.level_all[l].p, (int)pl.level_all[l].n);
        const int ge = ge_table(c, alpha_base * std::pow(4.0, l - bl));
        if (!c.subtract_non_leaf) fmm_apply(c, c.f_source_tmp, c.f_target_tmp, l, true, 1.0, IBLGF_IB2xIB, ge);
        launch_axpy_blocks(c, tt, c.field(tgt), pl.level_all[l].p, (int)pl.level_all[l].n, 1.0, true);
        return;
    }
    launch_axpy_blocks(c, c.field(src), st, pl.leaves.p, (int)pl.leaves.n, 1.0, true);
    for (int ls = depth - 2; ls >= bl; --ls) launch_tp_axes(c, pl.coarsify[ls], st, st, coarse_m, 0);
    // intrp_to_correction_buffer (poisson.hpp:1015-1069)
    for (int l = depth - 2; l >= bl; --l)
    {
        launch_halo(c, st, ol.list[l].p, (int)ol.list[l].n);
        launch_tp_axes(c, pl.corr_intrp[l], st, st, intrp_m, 2);
    }
    for (int l = bl; l < depth; ++l)
    {
        // LGF_GE::change_level_impl: alpha = alpha_base * 4^(l - base)
        const int ge = ge_table(c, alpha_base * std::pow(4.0, l - bl));
        fmm_apply(c, c.f_source_tmp, c.f_target_tmp, l, false, 1.0, IBLGF_AMR2AMR, ge);
        if (!c.subtract_non_leaf) fmm_apply(c, c.f_source_tmp, c.f_target_tmp, l, true, 1.0, IBLGF_AMR2AMR, ge);
        launch_axpy_blocks(c, tt, c.field(tgt), pl.level_all[l].p, (int)pl.level_all[l].n, 1.0, true);
    }
}

void poisson_release(Ctx& c)
{
    c.ext[Ctx::kExtPLists].reset();
    c.ext[Ctx::kExtOpLists].reset();
}

void poisson_apply_lgf(Ctx& c, int src, int tgt, int fmm_type)
{
    need_single(c);
    if (!c.finalized) throw Error(IBLGF_EINVAL, "domain not finalized");
    if (fmm_type < IBLGF_STREAM || fmm_type > IBLGF_IB2AMR) throw Error(IBLGF_EINVAL, "unknown fmm_type");
    PoissonLists& pl = poisson_lists(c);
    double* st = c.field(c.f_source_tmp);
    double* tt = c.field(c.f_target_tmp);
    double* ct = c.field(c.f_correction_tmp);
    const size_t bytes = c.field_elems() * sizeof(double);
    launch_fill_zero(c, st, bytes / sizeof(double));
    launch_fill_zero(c, tt, bytes / sizeof(double));
    launch_fill_zero(c, ct, bytes / sizeof(double));
    if (fmm_type == IBLGF_IB2AMR)
    {
        // finest-level interior copy, coarsified (cell mesh), one sweep per
        // level with the IB2AMR mask, leaves assigned, no source correction
        // (poisson.hpp:617-618, 632-634, 702-745)
        const int bl = c.tree.base_level, depth = c.tree.depth;
        launch_copy_interior(c, c.field(src), st, pl.level_all[depth - 1].p, (int)pl.level_all[depth - 1].n);
        for (int ls = depth - 2; ls >= bl; --ls) launch_tp(c, pl.coarsify[ls], st, st, 4, 0);
        for (int l = bl; l < depth && !c.subtract_non_leaf; ++l)
        {
            fmm_apply(c, c.f_source_tmp, c.f_target_tmp, l, false, 1.0, IBLGF_IB2AMR);
            launch_axpy_blocks(c, tt, c.field(tgt), pl.level_leaves[l].p, (int)pl.level_leaves[l].n, 1.0, true);
        }
        return;
    }
    if (fmm_type == IBLGF_xIB2IB || fmm_type == IBLGF_IB2xIB)
    {
        // finest level only: copy_level (interior), one sweep with the IB
        // mask, leaves of that level assigned (poisson.hpp:615-616, 702-745)
        const int l = c.tree.depth - 1;
        launch_copy_interior(c, c.field(src), st, pl.level_all[l].p, (int)pl.level_all[l].n);
        if (!c.subtract_non_leaf)
        {
            fmm_apply(c, c.f_source_tmp, c.f_target_tmp, l, false, 1.0, fmm_type);
            launch_axpy_blocks(c, tt, c.field(tgt), pl.level_leaves[l].p, (int)pl.level_leaves[l].n, 1.0, true);
        }
        return;
    }
    if (fmm_type == IBLGF_STREAM)
    {
        // base level only: copy_level (interior), one sweep with the stream
        // mask, leaves copied out (poisson.hpp:612-614, 749-781)
        const int bl = c.tree.base_level;
        launch_copy_interior(c, c.field(src), st, pl.level_all[bl].p, (int)pl.level_all[bl].n);
        if (!c.subtract_non_leaf)
        {
            fmm_apply(c, c.f_source_tmp, c.f_target_tmp, bl, false, 1.0, IBLGF_STREAM);
            launch_axpy_blocks(c, tt, c.field(tgt), pl.level_leaves[bl].p, (int)pl.level_leaves[bl].n, 1.0, true);
        }
        return;
    }
    launch_axpy_blocks(c, c.field(src), st, pl.leaves.p, (int)pl.leaves.n, 1.0, true);
    const int bl = c.tree.base_level, depth = c.tree.depth;
    for (int ls = depth - 2; ls >= bl; --ls) launch_tp(c, pl.coarsify[ls], st, st, 4, 0);
    for (int l = bl; l < depth; ++l)
    {
        if (!c.subtract_non_leaf)
        {
            fmm_apply(c, c.f_source_tmp, c.f_target_tmp, l, true, 1.0, IBLGF_AMR2AMR);
            launch_tp(c, pl.cc_intrp[l], tt, tt, 2, 2);
            fmm_apply(c, c.f_source_tmp, c.f_target_tmp, l, false, 1.0, IBLGF_AMR2AMR);
            launch_axpy_blocks(c, tt, c.field(tgt), pl.level_leaves[l].p, (int)pl.level_leaves[l].n, 1.0, true);
        }
        if (!c.use_correction || l == depth - 1) continue;
        launch_halo(c, st, pl.level_all[l].p, (int)pl.level_all[l].n);
        launch_tp(c, pl.corr_intrp[l], st, ct, 2, 2);
        const double dx = c.cfg.dx_base / std::pow(2.0, l - bl) / 2.0;
        launch_source_correction(c, tt, ct, pl.children[l].p, (int)pl.children[l].n, 1.0 / (dx * dx));
        launch_axpy_blocks(c, ct, st, pl.level_all[l + 1].p, (int)pl.level_all[l + 1].n, 1.0, false);
    }
}

}  // namespace iblgf_b200
