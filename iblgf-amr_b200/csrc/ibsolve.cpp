// Immersed-boundary force solve on the device:
//   points, flags and influence lists: IB::init / ib_block_overlap /
//     yang3 (include/iblgf/domain/ib.hpp:70-120, 652-705),
//     ServerBase::update_ib_flag (domain/decomposition/server.hpp:544-576),
//     Client::update_ib_rank_and_infl (client.hpp:1262-1320)
//   masks: FmmMaskBuilder IB2xIB / xIB2IB / IB2AMR (fmm/fmm.hpp:70-190)
//   solve: LinSysSolver::ib_solve, CG_solve, ET_H_S_E, apply_Schur,
//     projection, smearing (solver/linsys/linsys.hpp:113-450)
// The delta weights of every (point, influence node, component) are computed
// here once; projection and smearing run as deterministic device gathers. The
// Schur operator's divergence, masked LGF solve, gradient and integrating
// factor are the library's own kernels on device fields. CG vectors and dot
// products are FP64 on the host (3 n values per iteration).
#include <algorithm>
#include <cmath>
#include <functional>
#include <map>
#include <memory>
#include <random>

#include "ctx.hpp"

namespace iblgf_b200
{
void launch_axpby(Ctx& c, double* to, const double* from, double a, int mode);

namespace
{
double yang3(double x)
{
    const double r = std::fabs(x);
    if (r > 2) return 0.0;
    const double r2 = r * r, s3 = std::sqrt(3.0);
    if (r <= 1.0)
        return 17.0 / 48.0 + s3 * M_PI / 108.0 + r / 4.0 - r2 / 4.0 +
               (1.0 - 2.0 * r) / 16 * std::sqrt(-12.0 * r2 + 12.0 * r + 1.0) -
               s3 / 12.0 * std::asin(s3 / 2.0 * (2.0 * r - 1.0));
    return 55.0 / 48.0 - s3 * M_PI / 108.0 - 13.0 * r / 12.0 + r2 / 4.0 +
           (2.0 * r - 3.0) / 48.0 * std::sqrt(-12.0 * r2 + 36.0 * r - 23.0) +
           s3 / 36.0 * std::asin(s3 / 2.0 * (2 * r - 3.0));
}

// learned warm start (see warmstart.cu): samples of the first train_steps
// steps, then a network trained on them predicts f0 - f_prev per stage
struct WarmStart
{
    // 0: previous step's force of the stage (the reference), 1: learned
    // correction on top of the previous force, 2: linear extrapolation
    // 2 f_prev - f_prev2 (f_prev until two forces exist)
    int mode = 0;
    int train_steps = 0, epochs = 0, steps_seen = 0, n_params = 0;
    float lr = 1e-3f;
    unsigned seed = 1;
    bool trained = false;
    float loss_first = 0.0f, loss_last = 0.0f;
    // samples (stage, rhs change, previous force, its last change, target
    // f - f_prev) and per-stage input / target scales
    std::vector<int> s_stage;
    std::vector<std::vector<double>> s_duc, s_fprev, s_dfp, s_t;
    float sb[4] = {1, 1, 1, 1}, sf[4] = {1, 1, 1, 1}, sd[4] = {1, 1, 1, 1}, st[4] = {1, 1, 1, 1};
    std::vector<double> uc_prev[4];  // right-hand side of the previous step per stage
    int count_host[4] = {0, 0, 0, 0};  // forces recorded per stage (host mirror of fcount)
    std::vector<int> order;  // network position -> IB point (Morton order)
    DevBuf<float> params, grads, m, v, x, t, h1, h2, y, dy, dh1, dh2, partial;
};

struct IbState
{
    int n = 0;
    double Re = 0.0;
    std::vector<double> X;
    std::vector<int> flags;  // per octant: bit0 is_ib (parents of IB blocks included), bit1 is_extended_ib
    // projection: per point CSR over entries (field offset, 3 weights)
    DevBuf<int> ptr;
    DevBuf<long long> at;
    DevBuf<double> w;
    // smearing: per node CSR over (point, entry)
    DevBuf<long long> node_at;
    DevBuf<int> nptr, npt, nent;
    int n_nodes = 0;
    // face-plane cleaning at the finest level: IB region (width 2) and the
    // operator's correction-boundary clean (width 2)
    DevBuf<int> ibc_list, cb_list, corr_list;
    DevBuf<unsigned char> ibc_faces, cb_faces;
    int n_ibc = 0, n_cb = 0, n_corr = 0;
    bool clean_base = false;
    int face_aux[3] = {-1, -1, -1}, face_aux2[3] = {-1, -1, -1}, cell_aux2 = -1;
    // force CG of LinSysSolver::CG_solve on the device: iterate, residual,
    // direction, Schur product, projected velocity (3 n each), the scalars
    // [rsold, p.Ap, rsnew, f.f] and controls [done, iterations, not converged]
    DevBuf<double> cg_f, cg_r, cg_p, cg_Ap, cg_uc, cg_sc;
    DevBuf<int> cg_ctl;
    DevBuf<int> cg_rec;                 // per stage 0..3: [iterations, not converged] of its last solve
    DevBuf<double> fprev[4];            // IB::force_prev per IF-HERK stage (CG warm start), on the device
    DevBuf<double> fprev2[4];           // the stage's force one step further back
    DevBuf<int> fcount;                 // forces recorded per stage (extrapolation needs two)
    int* done_host = nullptr;           // pinned: the done flag, read once per iteration of a direct solve
    cudaStream_t body_stream = nullptr; // captures the loop body of a solve inside a graph
    WarmStart ws;
    IbState() = default;
    IbState(const IbState&) = delete;
    IbState& operator=(const IbState&) = delete;
    ~IbState()
    {
        if (done_host) cudaFreeHost(done_host);
        if (body_stream) cudaStreamDestroy(body_stream);
    }
};

// face neighbour direction -> face bit (0 z-, 1 y-, 2 x-, 3 x+, 4 y+, 5 z+)
int face_bit(int i)
{
    switch (i)
    {
        case 4: return 0;
        case 10: return 1;
        case 12: return 2;
        case 14: return 3;
        case 16: return 4;
        case 22: return 5;
        default: return -1;
    }
}

IbState& state(Ctx& c)
{
    auto* s = c.ext_get<IbState>(Ctx::kExtIb);
    if (!s) throw Error(IBLGF_EINVAL, "no immersed-boundary points set");
    return *s;
}
}  // namespace

void ib_set_points(Ctx& c, int n, const double* X, double Re)
{
    need_single(c);
    if (!c.finalized) throw Error(IBLGF_EINVAL, "domain not finalized");
    if (n <= 0 || !X) throw Error(IBLGF_EINVAL, "no points");
    if (!(Re > 0)) throw Error(IBLGF_EINVAL, "Re must be positive");
    auto s = std::make_unique<IbState>();
    s->n = n;
    s->Re = Re;
    s->X.assign(X, X + 3 * (size_t)n);
    const int l_max = c.tree.depth - 1, bl = c.tree.base_level;
    const int ib_level = l_max - bl;
    const int e = c.cfg.block_extent, Nb = c.Nb;
    const double dx_base = c.cfg.dx_base;
    const double dx_ib = dx_base / std::pow(2, ib_level);
    const double ddf_radius = 4.5, safety = 5.0 / (Re * dx_ib) + 1.0;
    auto overlap = [&](int i, int o, int radius_level) {
        double r = 0;
        if (radius_level == 2) r = ddf_radius + safety + 10.0;
        else if (radius_level == 1) r = ddf_radius + 5.0;
        const double sc = std::pow(2, ib_level - (c.levels[o] - bl));
        const double factor = std::pow(2, ib_level) / dx_base;
        for (int q = 0; q < 3; ++q)
        {
            const double base = c.bbase[3 * o + q] * sc - r;
            const double mx = base + e * sc + 2 * r - 1;
            if (mx + 1 < X[3 * i + q] * factor || base >= X[3 * i + q] * factor) return false;
        }
        return true;
    };
    s->flags.assign(c.n_oct, 0);
    for (int i = 0; i < n; ++i)
        for (int o : c.level_octs[l_max])
            if (overlap(i, o, 2))
            {
                s->flags[o] |= 2;
                if (overlap(i, o, 1) && (c.flags[o] & 1)) s->flags[o] |= 1;
            }
    std::vector<int> ibm = s->flags;
    build_ib_masks(c, ibm);
    s->flags = ibm;
    // influence lists / nodes / weights (client.hpp:1262-1320, operators.hpp:841-861)
    std::vector<int> ptr{0};
    std::vector<long long> at;
    std::vector<double> w;
    std::vector<int> ent_pt;
    const size_t B = c.block_elems();
    for (int i = 0; i < n; ++i)
    {
        for (int o : c.level_octs[l_max])
        {
            if (!(c.flags[o] & 1) || !overlap(i, o, 1)) continue;
            const double sc = std::pow(2, c.levels[o] - bl) / dx_base;
            for (int k = 0; k < e; ++k)
                for (int j = 0; j < e; ++j)
                    for (int a = 0; a < e; ++a)
                    {
                        const int nd[3] = {c.bbase[3 * o] + a, c.bbase[3 * o + 1] + j, c.bbase[3 * o + 2] + k};
                        double dist[3];
                        bool in = true;
                        for (int q = 0; q < 3; ++q)
                        {
                            dist[q] = nd[q] - X[3 * i + q] * sc;
                            if (std::fabs(dist[q]) >= ddf_radius + 1.0) in = false;
                        }
                        if (!in) continue;
                        at.push_back((long long)o * B + (a + 1) + (size_t)Nb * ((j + 1) + (size_t)Nb * (k + 1)));
                        for (int cc = 0; cc < 3; ++cc)
                            w.push_back(yang3(dist[0] + (cc == 0 ? 0.0 : 0.5)) *
                                        yang3(dist[1] + (cc == 1 ? 0.0 : 0.5)) *
                                        yang3(dist[2] + (cc == 2 ? 0.0 : 0.5)));
                        ent_pt.push_back(i);
                    }
        }
        ptr.push_back((int)at.size());
    }
    // node-major view for the smearing gather, points in increasing order
    std::map<long long, std::vector<int>> by_node;
    for (size_t e_ = 0; e_ < at.size(); ++e_) by_node[at[e_]].push_back((int)e_);
    std::vector<long long> node_at;
    std::vector<int> nptr{0}, npt, nent;
    for (auto& kv : by_node)
    {
        node_at.push_back(kv.first);
        for (int e_ : kv.second)
        {
            npt.push_back(ent_pt[e_]);
            nent.push_back(e_);
        }
        nptr.push_back((int)npt.size());
    }
    s->ptr.upload(ptr, c.stream);
    s->at.upload(at, c.stream);
    s->w.upload(w, c.stream);
    s->node_at.upload(node_at, c.stream);
    s->nptr.upload(nptr, c.stream);
    s->npt.upload(npt, c.stream);
    s->nent.upload(nent, c.stream);
    s->n_nodes = (int)node_at.size();
    // face-plane cleaning lists at the finest level
    std::vector<int> ibc_list, cb_list, corr;
    std::vector<unsigned char> ibc_faces, cb_faces;
    for (int o : c.level_octs[l_max])
    {
        unsigned char m1 = 0, m2 = 0;
        for (int i = 0; i < 27; ++i)
        {
            const int b = face_bit(i);
            if (b < 0) continue;
            const int q = c.nbr[27 * (size_t)o + i];
            if (q < 0 || !(ibm[q] & 1)) m1 |= (unsigned char)(1u << b);
            if (q < 0 || (c.flags[q] & 2)) m2 |= (unsigned char)(1u << b);
        }
        if (m1)
        {
            ibc_list.push_back(o);
            ibc_faces.push_back(m1);
        }
        if (m2)
        {
            cb_list.push_back(o);
            cb_faces.push_back(m2);
        }
        if (c.flags[o] & 2) corr.push_back(o);
    }
    s->clean_base = l_max == bl;
    s->ibc_list.upload(ibc_list, c.stream);
    s->ibc_faces.upload(ibc_faces, c.stream);
    s->cb_list.upload(cb_list, c.stream);
    s->cb_faces.upload(cb_faces, c.stream);
    s->corr_list.upload(corr, c.stream);
    s->n_ibc = (int)ibc_list.size();
    s->n_cb = (int)cb_list.size();
    s->n_corr = (int)corr.size();
    if (const IbState* old = c.ext_get<IbState>(Ctx::kExtIb))
    {
        for (int k = 0; k < 3; ++k)
        {
            s->face_aux[k] = old->face_aux[k];
            s->face_aux2[k] = old->face_aux2[k];
        }
        s->cell_aux2 = old->cell_aux2;
    }
    else
    {
        for (int k = 0; k < 3; ++k)
        {
            s->face_aux[k] = field_create(c);
            s->face_aux2[k] = field_create(c);
        }
        s->cell_aux2 = field_create(c);
    }
    for (DevBuf<double>* b : {&s->cg_f, &s->cg_r, &s->cg_p, &s->cg_Ap, &s->cg_uc}) b->alloc(3 * (size_t)n);
    for (int k = 0; k < 4; ++k)
        for (DevBuf<double>* fp : {&s->fprev[k], &s->fprev2[k]})
        {
            fp->alloc(3 * (size_t)n);
            launch_fill_zero(c, fp->p, fp->n);
        }
    s->fcount.upload(std::vector<int>(4, 0), c.stream);
    s->cg_sc.upload(std::vector<double>(4, 0.0), c.stream);
    s->cg_ctl.upload(std::vector<int>(3, 0), c.stream);
    s->cg_rec.upload(std::vector<int>(8, 0), c.stream);
    IBLGF_CUDA(cudaMallocHost(&s->done_host, sizeof(int)));
    IBLGF_CUDA(cudaStreamCreateWithFlags(&s->body_stream, cudaStreamNonBlocking));
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    c.ext[Ctx::kExtIb] = std::shared_ptr<IbState>(std::move(s));
}

void ib_flags(Ctx& c, int* flags)
{
    IbState& s = state(c);
    for (int o = 0; o < c.n_oct; ++o) flags[o] = s.flags[o];
}

namespace
{
// Operator::ib_projection into the device vector out (3 n)
void projection(Ctx& c, IbState& s, const int* u, double* out)
{
    const double* pu[3] = {c.field(u[0]), c.field(u[1]), c.field(u[2])};
    launch_ib_projection(c, pu, s.ptr.p, s.at.p, s.w.p, s.n, out);
}

std::vector<double> download(Ctx& c, const double* d, size_t n)
{
    std::vector<double> h(n);
    IBLGF_CUDA(cudaMemcpyAsync(h.data(), d, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    return h;
}

// Operator::ib_smearing of the device forces f (3 n)
void smearing(Ctx& c, IbState& s, const double* f, const int* u, bool cleaning = true)
{
    double* pu[3] = {c.field(u[0]), c.field(u[1]), c.field(u[2])};
    if (cleaning)
        for (int k = 0; k < 3; ++k) launch_fill_zero(c, pu[k], c.field_elems());
    launch_ib_smearing(c, pu, s.node_at.p, s.nptr.p, s.npt.p, s.nent.p, s.w.p, s.n_nodes, f);
}

// apply_Schur<Source, Target>(xIB2IB), linsys.hpp:299-330
void apply_schur(Ctx& c, IbState& s, const int* src, const int* tgt)
{
    OpLists& ol = op_lists(c);
    const int l = c.tree.depth - 1;
    for (int k = 0; k < 3; ++k) launch_halo(c, c.field(src[k]), ol.list[l].p, (int)ol.list[l].n);
    const double* pin[3] = {c.field(src[0]), c.field(src[1]), c.field(src[2])};
    double* pc[1] = {c.field(s.cell_aux2)};
    launch_op(c, 2, pin, 3, pc, 1, ol.list[l].p, ol.dx[l].p, (int)ol.list[l].n, 1.0);
    // Operator::clean_leaf_correction_boundary<cell_aux2>(l, true, 2)
    launch_zero_blocks(c, pc[0], s.corr_list.p, s.n_corr);
    if (s.clean_base) launch_face_planes(c, pc[0], s.cb_list.p, s.cb_faces.p, s.n_cb, 2);
    launch_face_planes(c, pc[0], s.ibc_list.p, s.ibc_faces.p, s.n_ibc, 2);
    poisson_apply_lgf(c, s.cell_aux2, s.cell_aux2, IBLGF_xIB2IB);
    const double* pg[1] = {c.field(s.cell_aux2)};
    double* pt[3] = {c.field(tgt[0]), c.field(tgt[1]), c.field(tgt[2])};
    launch_op(c, 1, pg, 1, pt, 3, ol.list[l].p, ol.dx[l].p, (int)ol.list[l].n, 1.0);
    for (int k = 0; k < 3; ++k)
    {
        launch_halo(c, pt[k], ol.list[l].p, (int)ol.list[l].n);
        launch_face_planes(c, pt[k], s.ibc_list.p, s.ibc_faces.p, s.n_ibc, 2);
    }
}

// LinSysSolver::ET_H_S_E (linsys.hpp:260-297): device forces in, device
// projection out
void et_h_s_e(Ctx& c, IbState& s, const double* fin, double* fout, double alpha)
{
    for (int k = 0; k < 3; ++k) launch_fill_zero(c, c.field(s.face_aux[k]), c.field_elems());
    smearing(c, s, fin, s.face_aux2);
    if (std::fabs(alpha) > 1e-14)
        for (int k = 0; k < 3; ++k)
        {
            int rp[3] = {1, 1, 1};
            rp[k] = 0;  // face component k
            apply_if(c, s.face_aux2[k], s.face_aux2[k], alpha, IBLGF_IB2xIB, rp);
        }
    apply_schur(c, s, s.face_aux2, s.face_aux);
    for (int k = 0; k < 3; ++k) launch_axpby(c, c.field(s.face_aux2[k]), c.field(s.face_aux[k]), -1.0, 1);
    projection(c, s, s.face_aux2, fout);
}
}  // namespace

bool ib_active(const Ctx& c) { return c.ext[Ctx::kExtIb] != nullptr; }

namespace
{
void ws_init(WarmStart& w, Ctx& c)
{
    int o[7];
    ws_offsets(o);
    w.n_params = o[6];
    std::vector<float> p(o[6], 0.0f);
    std::mt19937 rng(w.seed);
    const int C = kWsChannels;
    auto fill = [&](int a, int b, int fan_in, float gain) {
        std::uniform_real_distribution<float> U(-1.0f, 1.0f);
        const float bound = gain / std::sqrt((float)fan_in);
        for (int i = a; i < b; ++i) p[i] = bound * U(rng);
    };
    fill(o[0], o[1], kWsInputs * 5, std::sqrt(6.0f));
    fill(o[2], o[3], C * 5, std::sqrt(6.0f));
    fill(o[4], o[5], C * 5, 0.1f);
    w.params.upload(p, c.stream);
    std::vector<float> z(o[6], 0.0f);
    w.grads.upload(z, c.stream);
    w.m.upload(z, c.stream);
    w.v.upload(z, c.stream);
}

// x [S][9][N] = ((uc - uc_prev) / sb, f_prev / sf, (f_prev - f_prev2) / sd),
// points in network order
std::vector<float> ws_inputs(const WarmStart& w, const std::vector<int>& stage,
                             const std::vector<const std::vector<double>*>& duc,
                             const std::vector<const std::vector<double>*>& fp,
                             const std::vector<const std::vector<double>*>& dfp, int N)
{
    const int I = kWsInputs;
    std::vector<float> x(duc.size() * I * (size_t)N);
    for (size_t s_ = 0; s_ < duc.size(); ++s_)
    {
        const int st = stage[s_];
        for (int ch = 0; ch < 3; ++ch)
            for (int q = 0; q < N; ++q)
            {
                const int i = w.order[q];
                x[(s_ * I + ch) * N + q] = (float)((*duc[s_])[3 * i + ch] / w.sb[st]);
                x[(s_ * I + 3 + ch) * N + q] = (float)((*fp[s_])[3 * i + ch] / w.sf[st]);
                x[(s_ * I + 6 + ch) * N + q] = (float)((*dfp[s_])[3 * i + ch] / w.sd[st]);
            }
    }
    return x;
}

void ws_train(Ctx& c, WarmStart& w, int N)
{
    const int S = (int)w.s_duc.size();
    if (!S) return;
    // per-stage rms scales of the inputs and of the target
    for (int st = 1; st <= 3; ++st)
    {
        double sb = 0, sf = 0, sd = 0, stt = 0;
        long long cnt = 0;
        for (int s_ = 0; s_ < S; ++s_)
        {
            if (w.s_stage[s_] != st) continue;
            ++cnt;
            for (int i = 0; i < 3 * N; ++i)
            {
                sb += w.s_duc[s_][i] * w.s_duc[s_][i];
                sf += w.s_fprev[s_][i] * w.s_fprev[s_][i];
                sd += w.s_dfp[s_][i] * w.s_dfp[s_][i];
                stt += w.s_t[s_][i] * w.s_t[s_][i];
            }
        }
        const double m = cnt ? cnt * 3.0 * N : 1.0;
        auto scale = [&](double q) { return q > 0 ? (float)std::sqrt(q / m) : 1.0f; };
        w.sb[st] = scale(sb);
        w.sf[st] = scale(sf);
        w.sd[st] = scale(sd);
        w.st[st] = scale(stt);
    }
    std::vector<const std::vector<double>*> duc, fp, dfp;
    for (int s_ = 0; s_ < S; ++s_)
    {
        duc.push_back(&w.s_duc[s_]);
        fp.push_back(&w.s_fprev[s_]);
        dfp.push_back(&w.s_dfp[s_]);
    }
    std::vector<float> x = ws_inputs(w, w.s_stage, duc, fp, dfp, N), t(S * 3 * (size_t)N);
    for (int s_ = 0; s_ < S; ++s_)
        for (int ch = 0; ch < 3; ++ch)
            for (int q = 0; q < N; ++q)
            {
                const int i = w.order[q];
                t[((size_t)s_ * 3 + ch) * N + q] = (float)(w.s_t[s_][3 * i + ch] / w.st[w.s_stage[s_]]);
            }
    w.x.upload(x, c.stream);
    w.t.upload(t, c.stream);
    const size_t hs = (size_t)S * kWsChannels * N;
    w.h1.alloc(hs);
    w.h2.alloc(hs);
    w.dh1.alloc(hs);
    w.dh2.alloc(hs);
    w.y.alloc((size_t)S * 3 * N);
    w.dy.alloc((size_t)S * 3 * N);
    for (int ep = 0; ep < w.epochs; ++ep)
    {
        ws_forward(c, w.params.p, w.x.p, S, N, w.h1.p, w.h2.p, w.y.p);
        const float l = ws_backward(c, w.params.p, w.x.p, w.t.p, S, N, w.h1.p, w.h2.p, w.y.p, w.dy.p, w.dh2.p,
                                    w.dh1.p, w.grads.p, w.partial);
        if (ep == 0) w.loss_first = l;
        w.loss_last = l;
        ws_adam(c, w.params.p, w.grads.p, w.m.p, w.v.p, w.n_params, w.lr, ep + 1);
    }
    w.trained = true;
}

// f0 = f_base + st * net(...), f_base the previous force and st the stage's
// rms of f - f_base in the samples
std::vector<double> ws_predict(Ctx& c, WarmStart& w, int stage, const std::vector<double>& duc,
                               const std::vector<double>& fp, const std::vector<double>& dfp,
                               const std::vector<double>& fbase, int N)
{
    std::vector<float> x = ws_inputs(w, {stage}, {&duc}, {&fp}, {&dfp}, N);
    DevBuf<float> dx, h1, h2, y;
    dx.upload(x, c.stream);
    h1.alloc((size_t)kWsChannels * N);
    h2.alloc((size_t)kWsChannels * N);
    y.alloc(3 * (size_t)N);
    ws_forward(c, w.params.p, dx.p, 1, N, h1.p, h2.p, y.p);
    std::vector<float> hy(3 * (size_t)N);
    IBLGF_CUDA(cudaMemcpyAsync(hy.data(), y.p, hy.size() * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    std::vector<double> f0(fbase);
    for (int ch = 0; ch < 3; ++ch)
        for (int q = 0; q < N; ++q) f0[3 * w.order[q] + ch] += (double)w.st[stage] * hy[(size_t)ch * N + q];
    return f0;
}
}  // namespace

void ib_warmstart(Ctx& c, int mode, int train_steps, int epochs, double lr, unsigned seed)
{
    IbState& s = state(c);
    if (mode < 0 || mode > 2) throw Error(IBLGF_EINVAL, "warm-start mode must be 0, 1 or 2");
    if (mode == 1 && (train_steps <= 0 || epochs <= 0 || !(lr > 0)))
        throw Error(IBLGF_EINVAL, "learned warm start needs train_steps, epochs and lr > 0");
    WarmStart& w = s.ws;
    w = WarmStart();
    w.mode = mode;
    w.train_steps = train_steps;
    w.epochs = epochs;
    w.lr = (float)lr;
    w.seed = seed;
    // network order: Morton order of the points (10 bits per axis over their
    // bounding box), so that the convolution's neighbours are spatial ones
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < s.n; ++i)
        for (int q = 0; q < 3; ++q)
        {
            lo[q] = std::min(lo[q], s.X[3 * i + q]);
            hi[q] = std::max(hi[q], s.X[3 * i + q]);
        }
    std::vector<std::pair<unsigned long long, int>> key(s.n);
    for (int i = 0; i < s.n; ++i)
    {
        unsigned long long k = 0;
        unsigned v[3];
        for (int q = 0; q < 3; ++q)
        {
            const double span = hi[q] > lo[q] ? hi[q] - lo[q] : 1.0;
            v[q] = (unsigned)std::min(1023.0, std::floor((s.X[3 * i + q] - lo[q]) / span * 1023.0));
        }
        for (int b = 9; b >= 0; --b)
            for (int q = 2; q >= 0; --q) k = (k << 1) | ((v[q] >> b) & 1u);
        key[i] = {k, i};
    }
    std::sort(key.begin(), key.end());
    w.order.resize(s.n);
    for (int q = 0; q < s.n; ++q) w.order[q] = key[q].second;
    if (mode == 1) ws_init(w, c);
}

void ib_warmstart_info(Ctx& c, double* info)
{
    IbState& s = state(c);
    const WarmStart& w = s.ws;
    info[0] = w.mode;
    info[1] = w.trained ? 1 : 0;
    info[2] = (double)w.s_duc.size();
    info[3] = w.loss_first;
    info[4] = w.loss_last;
    info[5] = w.n_params;
}

void ws_check(Ctx& c, int S, int N, const float* params, const float* x, const float* tgt, float* y, float* grads,
              float* loss)
{
    int o[7];
    ws_offsets(o);
    DevBuf<float> dp, dx, dt, h1, h2, dy_, yy, dh1, dh2, g, part;
    dp.upload(std::vector<float>(params, params + o[6]), c.stream);
    dx.upload(std::vector<float>(x, x + (size_t)S * kWsInputs * N), c.stream);
    dt.upload(std::vector<float>(tgt, tgt + (size_t)S * 3 * N), c.stream);
    const size_t hs = (size_t)S * kWsChannels * N;
    h1.alloc(hs);
    h2.alloc(hs);
    dh1.alloc(hs);
    dh2.alloc(hs);
    yy.alloc((size_t)S * 3 * N);
    dy_.alloc((size_t)S * 3 * N);
    g.alloc(o[6]);
    ws_forward(c, dp.p, dx.p, S, N, h1.p, h2.p, yy.p);
    const float l = ws_backward(c, dp.p, dx.p, dt.p, S, N, h1.p, h2.p, yy.p, dy_.p, dh2.p, dh1.p, g.p, part);
    IBLGF_CUDA(cudaMemcpyAsync(y, yy.p, (size_t)S * 3 * N * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
    IBLGF_CUDA(cudaMemcpyAsync(grads, g.p, o[6] * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    *loss = l;
}

const int* ib_face_aux2(Ctx& c) { return state(c).face_aux2; }

namespace
{
// One iteration of CG_solve (linsys.hpp:202-229) on the device: Ap = S p,
// p.Ap, the update of f and r, r.r and f.f, the next direction and the
// scalar step; inside a graph's loop the last launch sets the loop condition
void cg_iteration(Ctx& c, IbState& s, double alpha, double threshold, int max_iter, unsigned long long cond,
                  bool set_cond)
{
    const int m = 3 * s.n;
    et_h_s_e(c, s, s.cg_p.p, s.cg_Ap.p, alpha);
    launch_cg_dot(c, s.cg_p.p, s.cg_Ap.p, nullptr, nullptr, m, s.cg_sc.p + 1, nullptr, s.cg_ctl.p);
    launch_cg_update(c, s.cg_f.p, s.cg_r.p, s.cg_p.p, s.cg_Ap.p, m, s.cg_sc.p, s.cg_ctl.p);
    launch_cg_dot(c, s.cg_r.p, s.cg_r.p, s.cg_f.p, s.cg_f.p, m, s.cg_sc.p + 2, s.cg_sc.p + 3, s.cg_ctl.p);
    launch_cg_direction(c, s.cg_p.p, s.cg_r.p, m, s.cg_sc.p, s.cg_ctl.p, threshold);
    launch_cg_advance(c, s.cg_sc.p, s.cg_ctl.p, threshold, max_iter, cond, set_cond);
}

// LinSysSolver::ib_solve + CG_solve (linsys.hpp:113-230) from the iterate
// already in cg_f; rec (device, 2 ints) receives [iterations, not converged].
// Outside a stream capture the host reads the done flag once per iteration;
// inside one the loop is a conditional while-node of the graph, its body one
// iteration, so a captured time step runs the whole solve on the device.
void cg_solve(Ctx& c, IbState& s, const int* u, double alpha, double threshold, int max_iter, int* rec)
{
    const int m = 3 * s.n;
    projection(c, s, u, s.cg_uc.p);
    for (int k = 0; k < 3; ++k) launch_fill_zero(c, c.field(s.face_aux2[k]), c.field_elems());
    et_h_s_e(c, s, s.cg_f.p, s.cg_Ap.p, alpha);
    launch_cg_init(c, s.cg_uc.p, s.cg_Ap.p, s.cg_r.p, s.cg_p.p, m, s.cg_ctl.p, max_iter);
    launch_cg_dot(c, s.cg_r.p, s.cg_r.p, nullptr, nullptr, m, s.cg_sc.p, nullptr, nullptr);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    IBLGF_CUDA(cudaStreamGetCaptureInfo(c.stream, &cs, nullptr, &g, &deps, &nd));
    if (cs == cudaStreamCaptureStatusActive)
    {
        cudaGraphConditionalHandle h;
        IBLGF_CUDA(cudaGraphConditionalHandleCreate(&h, g, max_iter > 0 ? 1u : 0u, cudaGraphCondAssignDefault));
        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        IBLGF_CUDA(cudaGraphAddNode(&node, g, deps, nd, &np));
        cudaGraph_t body = np.conditional.phGraph_out[0];
        IBLGF_CUDA(cudaStreamUpdateCaptureDependencies(c.stream, &node, 1, cudaStreamSetCaptureDependencies));
        IBLGF_CUDA(cudaStreamBeginCaptureToGraph(s.body_stream, body, nullptr, nullptr, 0,
                                                 cudaStreamCaptureModeRelaxed));
        cudaStream_t outer = c.stream;
        c.stream = s.body_stream;
        try
        {
            cg_iteration(c, s, alpha, threshold, max_iter, (unsigned long long)h, true);
        }
        catch (...)
        {
            c.stream = outer;
            cudaGraph_t dummy = nullptr;
            cudaStreamEndCapture(s.body_stream, &dummy);
            throw;
        }
        c.stream = outer;
        cudaGraph_t captured = nullptr;
        IBLGF_CUDA(cudaStreamEndCapture(s.body_stream, &captured));
    }
    else
    {
        for (int k = 0; k < max_iter; ++k)
        {
            cg_iteration(c, s, alpha, threshold, max_iter, 0, false);
            IBLGF_CUDA(cudaMemcpyAsync(s.done_host, s.cg_ctl.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
            IBLGF_CUDA(cudaStreamSynchronize(c.stream));
            if (*s.done_host) break;
        }
    }
    launch_cg_record(c, s.cg_ctl.p, rec);
}
}  // namespace

bool ib_graphable(const Ctx& c)
{
    const IbState* s = c.ext_get<IbState>(Ctx::kExtIb);
    return !s || s->ws.mode != 1;
}

// lin_sys_with_ib_solve's IB part (ifherk.hpp:1474-1494) after face_aux2 =
// r_i - grad d_i (+ IF): CG warm-started from the stage's previous force,
// pressure correction of d, then face_aux = grad d + E f (the caller
// subtracts it from r_i). With the reference warm start everything stays on
// the device; the learned warm start assembles its inputs on the host.
void ns_ib_stage(Ctx& c, int stage, double alpha, double threshold, int max_iter, int d_field, const int* face_aux,
                 const std::function<void()>& gradient_d, bool write_prev)
{
    IbState& s = state(c);
    WarmStart& w = s.ws;
    const size_t m = 3 * (size_t)s.n;
    int* rec = s.cg_rec.p + 2 * stage;
    if (w.mode == 1 && write_prev)
    {
        projection(c, s, s.face_aux2, s.cg_uc.p);
        launch_ws_base(c, s.cg_f.p, s.fprev[stage].p, s.fprev2[stage].p, (int)m, s.fcount.p + stage, false);
        std::vector<double> uc = download(c, s.cg_uc.p, m), fp = download(c, s.fprev[stage].p, m),
                            fp2 = download(c, s.fprev2[stage].p, m), fbase = download(c, s.cg_f.p, m);
        std::vector<double> duc(uc), dfp(fp);
        if (!w.uc_prev[stage].empty())
            for (size_t i = 0; i < duc.size(); ++i) duc[i] -= w.uc_prev[stage][i];
        for (size_t i = 0; i < dfp.size(); ++i) dfp[i] -= fp2[i];
        const bool history = w.count_host[stage] >= 1 && !w.uc_prev[stage].empty();
        if (w.trained && history)
        {
            const std::vector<double> f0 = ws_predict(c, w, stage, duc, fp, dfp, fbase, s.n);
            IBLGF_CUDA(cudaMemcpyAsync(s.cg_f.p, f0.data(), m * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        }
        cg_solve(c, s, s.face_aux2, alpha, threshold, max_iter, rec);
        // samples from steps that have a previous force and right-hand side
        if (!w.trained && history)
        {
            std::vector<double> t = download(c, s.cg_f.p, m);
            for (size_t i = 0; i < t.size(); ++i) t[i] -= fbase[i];
            w.s_stage.push_back(stage);
            w.s_duc.push_back(duc);
            w.s_fprev.push_back(fp);
            w.s_dfp.push_back(dfp);
            w.s_t.push_back(t);
            if (stage == 3 && ++w.steps_seen >= w.train_steps) ws_train(c, w, s.n);
        }
        w.uc_prev[stage] = uc;
    }
    else
    {
        launch_ws_base(c, s.cg_f.p, s.fprev[stage].p, s.fprev2[stage].p, (int)m, s.fcount.p + stage, w.mode == 2);
        cg_solve(c, s, s.face_aux2, alpha, threshold, max_iter, rec);
    }
    if (write_prev)
    {
        launch_ws_record(c, s.fprev2[stage].p, s.fprev[stage].p, s.cg_f.p, (int)m, s.fcount.p + stage);
        ++w.count_host[stage];
    }
    // LinSysSolver::pressure_correction (linsys.hpp:131-145)
    OpLists& ol = op_lists(c);
    const int l = c.tree.depth - 1;
    launch_fill_zero(c, c.field(s.cell_aux2), c.field_elems());
    smearing(c, s, s.cg_f.p, s.face_aux2);
    for (int k = 0; k < 3; ++k) launch_halo(c, c.field(s.face_aux2[k]), ol.list[l].p, (int)ol.list[l].n);
    const double* pin[3] = {c.field(s.face_aux2[0]), c.field(s.face_aux2[1]), c.field(s.face_aux2[2])};
    double* pc[1] = {c.field(s.cell_aux2)};
    launch_op(c, 2, pin, 3, pc, 1, ol.list[l].p, ol.dx[l].p, (int)ol.list[l].n, 1.0);
    launch_zero_blocks(c, pc[0], s.corr_list.p, s.n_corr);
    if (s.clean_base) launch_face_planes(c, pc[0], s.cb_list.p, s.cb_faces.p, s.n_cb, 2);
    poisson_apply_lgf(c, s.cell_aux2, s.cell_aux2, IBLGF_IB2AMR);
    launch_axpby(c, c.field(d_field), c.field(s.cell_aux2), -1.0, 1);
    gradient_d();
    smearing(c, s, s.cg_f.p, face_aux, false);
}

void ib_force(Ctx& c, int stage, double* out, int* iters, int* not_converged)
{
    IbState& s = state(c);
    if (stage < 1 || stage > 3) throw Error(IBLGF_EINVAL, "stage must be 1, 2 or 3");
    if (out)
    {
        const std::vector<double> f = download(c, s.fprev[stage].p, 3 * (size_t)s.n);
        std::copy(f.begin(), f.end(), out);
    }
    int rec[2] = {0, 0};
    IBLGF_CUDA(cudaMemcpyAsync(rec, s.cg_rec.p + 2 * stage, sizeof(rec), cudaMemcpyDeviceToHost, c.stream));
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    if (iters) *iters = rec[0];
    if (not_converged) *not_converged = rec[1];
}

bool ib_solve(Ctx& c, const int* u, double alpha, double threshold, int max_iter, double* f, int* iters)
{
    IbState& s = state(c);
    const int nf = (int)c.fields.size();
    for (int k = 0; k < 3; ++k)
        if (u[k] < 0 || u[k] >= nf) throw Error(IBLGF_EINVAL, "bad velocity field id");
    const size_t m = 3 * (size_t)s.n;
    IBLGF_CUDA(cudaMemcpyAsync(s.cg_f.p, f, m * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    cg_solve(c, s, u, alpha, threshold, max_iter, s.cg_rec.p);  // record slot 0: direct solves
    IBLGF_CUDA(cudaMemcpyAsync(f, s.cg_f.p, m * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    int rec[2] = {0, 0};
    IBLGF_CUDA(cudaMemcpyAsync(rec, s.cg_rec.p, sizeof(rec), cudaMemcpyDeviceToHost, c.stream));
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    if (iters) *iters = rec[0];
    return rec[1] == 0;
}

void ib_release(Ctx& c) { c.ext[Ctx::kExtIb].reset(); }

std::vector<int> ib_octant_flags(Ctx& c)
{
    const IbState* s = c.ext_get<IbState>(Ctx::kExtIb);
    if (!s) return {};
    return s->flags;
}

// After an adaptation the point set is re-attached to the new tree (flags,
// masks, influence lists, cleaning lists); the stage forces and the warm-start
// network carry over
void ib_on_adapt(Ctx& c)
{
    IbState* old = c.ext_get<IbState>(Ctx::kExtIb);
    if (!old) return;
    std::vector<double> fp[4], fp2[4];
    for (int k = 0; k < 4; ++k)
    {
        fp[k] = download(c, old->fprev[k].p, old->fprev[k].n);
        fp2[k] = download(c, old->fprev2[k].p, old->fprev2[k].n);
    }
    std::vector<int> cnt(4);
    IBLGF_CUDA(cudaMemcpyAsync(cnt.data(), old->fcount.p, 4 * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    WarmStart ws = std::move(old->ws);
    const std::vector<double> X = old->X;
    const double Re = old->Re;
    ib_set_points(c, (int)(X.size() / 3), X.data(), Re);
    IbState& s = state(c);
    for (int k = 0; k < 4; ++k)
    {
        s.fprev[k].upload(fp[k], c.stream);
        s.fprev2[k].upload(fp2[k], c.stream);
    }
    s.fcount.upload(cnt, c.stream);
    IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    s.ws = std::move(ws);
}

}  // namespace iblgf_b200
