// ORACLE (test infrastructure): plain C entry points used by tests/ (ctypes),
// __graft_entry__.smoke() and bench.py's cpu_baseline leg.
#include <cstring>
#include <exception>
#include <memory>
#include <string>

#include "orc.hpp"

using namespace orc;

namespace
{
thread_local std::string g_err;
struct Handle
{
    std::unique_ptr<Domain> d;
    std::unique_ptr<Solver> s;
    // last adaptation: old canonical index per new octant (-1: new), the
    // interpolation parents (new canonical indices, in order)
    std::vector<int> adapt_src, adapt_parents;
    int adapt_old_n = 0;
    // IF-HERK state kept across orc_ns_step calls (the device keeps it per context)
    double ns_T_last = 0.0;
    bool ns_force_refresh = false;
};
template<class F>
int guard(F&& f)
{
    try
    {
        f();
        return 0;
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return 1;
    }
}
}  // namespace

extern "C" {

int orc_apply_lgf_type(void* hp, const double* src, double* tgt, int use_correction, int subtract_non_leaf,
                       int fmm_type);

const char* orc_last_error() { return g_err.c_str(); }

double orc_lgf_get(int x, int y, int z) { return lgf_get(x, y, z); }

int orc_lgf_table_size() { return lgf_table_size(); }

void orc_lgf_table(double* out) { std::memcpy(out, lgf_table().data(), sizeof(double) * lgf_table().size()); }

void orc_bessel_ie(double x, int nmax, double* out) { bessel_ie_all(x, nmax, out); }

void orc_nli_matrix(int Nb, int pts_cap, double* out) { nli_matrix(Nb, pts_cap, out); }

void orc_cc_matrix(int Nb, int pts_cap, int relpos, double* out) { cc_matrix(Nb, pts_cap, relpos, out); }

void* orc_domain_create(const int* bd_base, const int* bd_extent, int block_extent, double dx_base,
                        int n_blocks, const int* block_base, const int* block_ext)
{
    auto* h = new Handle;
    if (guard([&] {
            h->d = domain_create(bd_base, bd_extent, block_extent, dx_base, n_blocks, block_base,
                                 block_ext);
        }))
    {
        delete h;
        return nullptr;
    }
    return h;
}

void orc_domain_destroy(void* h) { delete static_cast<Handle*>(h); }

int orc_domain_init_refine(void* hp, int nRef, int global_refinement, RefinePred pred, void* user)
{
    auto* h = static_cast<Handle*>(hp);
    return guard([&] { h->d->init_refine(nRef, global_refinement, pred, user); });
}

// canonical order, masks (AMR2AMR for every refinement level, STREAM)
int orc_domain_finalize(void* hp, int subtract_non_leaf)
{
    auto* h = static_cast<Handle*>(hp);
    return guard([&] {
        h->d->construct_level_maps();
        h->d->construct_lists();
        h->d->finalize();
        fmm_lgf_mask_build(*h->d, subtract_non_leaf != 0);
        fmm_stream_mask_build(*h->d);
    });
}

// Domain::adapt (one process): tree change, new canonical order and masks.
// *n_octants gets the new octant count; fields follow with orc_adapt_field.
int orc_adapt(void* hp, int n_att, const unsigned long long* keys, const int* lchange, int subtract_non_leaf,
              int* base_mesh_update, int* n_octants)
{
    auto* h = static_cast<Handle*>(hp);
    return guard([&] {
        std::vector<std::pair<u64, int>> att(n_att);
        for (int i = 0; i < n_att; ++i) att[i] = {(u64)keys[i], lchange[i]};
        h->adapt_old_n = (int)h->d->octs.size();
        bool bmu = false;
        const std::vector<Octant*> parents = h->d->adapt(att, bmu);
        std::map<Octant*, int> old;
        h->d->construct_level_maps();
        for (auto& lm : h->d->level_maps)
            for (auto& kv : lm) old[kv.second] = kv.second->idx;
        h->d->construct_lists();
        h->d->finalize();
        h->adapt_src.assign(h->d->octs.size(), -1);
        for (Octant* o : h->d->octs) h->adapt_src[o->idx] = old[o];
        h->adapt_parents.clear();
        for (Octant* p : parents) h->adapt_parents.push_back(p->idx);
        for (Octant* o : h->d->octs)
            for (auto& m : o->mask) m = {false, false};
        fmm_lgf_mask_build(*h->d, subtract_non_leaf != 0);
        fmm_stream_mask_build(*h->d);
        *base_mesh_update = bmu ? 1 : 0;
        *n_octants = (int)h->d->octs.size();
        h->ns_force_refresh = h->ns_force_refresh || bmu;
    });
}

// one component field through the last adaptation: old (old octant count x
// Nb^3) -> out (new count x Nb^3); mesh >= 0 (0 cell, 1 face, 2 edge, with
// component comp) also interpolates each parent into all its children
// (cell_center_nli_intrp.hpp:310-420)
int orc_adapt_field(void* hp, const double* old, int mesh, int comp, double* out)
{
    auto* h = static_cast<Handle*>(hp);
    return guard([&] {
        const size_t B = (size_t)h->d->Nb * h->d->Nb * h->d->Nb;
        const size_t n = h->d->octs.size();
        Field f(n * B, 0.0);
        for (size_t i = 0; i < n; ++i)
            if (h->adapt_src[i] >= 0) std::copy(old + h->adapt_src[i] * B, old + (h->adapt_src[i] + 1) * B, &f[i * B]);
        if (mesh >= 0)
        {
            int rp[3];
            mesh_relpos(mesh, comp, rp);
            for (int pi : h->adapt_parents)
            {
                Octant* p = h->d->octs[pi];
                for (int c = 0; c < 8; ++c)
                {
                    Octant* ch = p->child[c].get();
                    if (!ch || !ch->has_data) continue;
                    h->s->cc_intrp_child(f, p, c, rp);
                }
            }
        }
        std::copy(f.begin(), f.end(), out);
    });
}

int orc_domain_info(void* hp, int* base_level, int* depth, int* n_octants)
{
    auto* h = static_cast<Handle*>(hp);
    *base_level = h->d->base_level;
    *depth = h->d->depth;
    *n_octants = (int)h->d->octs.size();
    return 0;
}

// flags: bit0 leaf, bit1 correction
int orc_domain_octants(void* hp, unsigned long long* keys, int* levels, int* flags, int* bbase)
{
    auto* h = static_cast<Handle*>(hp);
    for (size_t i = 0; i < h->d->octs.size(); ++i)
    {
        Octant* o = h->d->octs[i];
        keys[i] = o->key;
        levels[i] = o->level;
        flags[i] = (o->leaf ? 1 : 0) | (o->correction ? 2 : 0);
        for (int d = 0; d < 3; ++d) bbase[3 * i + d] = o->bbase[d];
    }
    return 0;
}

// neighbour (27 per octant) and influence (189 per octant) lists as canonical
// indices, -1 for absent
int orc_domain_lists(void* hp, int* nbr, int* infl, int* n_infl)
{
    auto* h = static_cast<Handle*>(hp);
    for (size_t i = 0; i < h->d->octs.size(); ++i)
    {
        Octant* o = h->d->octs[i];
        for (int j = 0; j < 27; ++j) nbr[27 * i + j] = o->neighbor[j] ? o->neighbor[j]->idx : -1;
        for (int j = 0; j < 189; ++j)
            infl[189 * i + j] = (j < o->n_infl && o->influence[j]) ? o->influence[j]->idx : -1;
        n_infl[i] = o->n_infl;
    }
    return 0;
}

int orc_domain_masks(void* hp, int mask_idx, unsigned char* out)
{
    auto* h = static_cast<Handle*>(hp);
    for (size_t i = 0; i < h->d->octs.size(); ++i)
    {
        out[2 * i] = h->d->octs[i]->mask[mask_idx][0];
        out[2 * i + 1] = h->d->octs[i]->mask[mask_idx][1];
    }
    return 0;
}

int orc_solver_create(void* hp, int intrp_order)
{
    auto* h = static_cast<Handle*>(hp);
    return guard([&] { h->s = std::make_unique<Solver>(h->d.get(), intrp_order); });
}

int orc_fmm_apply(void* hp, const double* src, double* tgt, int level, int nlas, double scale,
                  int fmm_type)
{
    auto* h = static_cast<Handle*>(hp);
    return guard([&] {
        const size_t n = h->d->octs.size() * (size_t)h->d->Nb * h->d->Nb * h->d->Nb;
        Field s(src, src + n), t(tgt, tgt + n);
        h->s->fmm_apply(s, t, level, nlas != 0, scale, fmm_type);
        std::memcpy(tgt, t.data(), n * sizeof(double));
    });
}

int orc_apply_lgf(void* hp, const double* src, double* tgt, int use_correction, int subtract_non_leaf)
{
    return orc_apply_lgf_type(hp, src, tgt, use_correction, subtract_non_leaf, AMR2AMR);
}

int orc_apply_lgf_type(void* hp, const double* src, double* tgt, int use_correction, int subtract_non_leaf,
                       int fmm_type)
{
    auto* h = static_cast<Handle*>(hp);
    return guard([&] {
        const size_t n = h->d->octs.size() * (size_t)h->d->Nb * h->d->Nb * h->d->Nb;
        Field s(src, src + n), t(tgt, tgt + n);
        h->s->apply_lgf(s, t, fmm_type, use_correction != 0, subtract_non_leaf != 0);
        std::memcpy(tgt, t.data(), n * sizeof(double));
    });
}

int orc_apply_if(void* hp, const double* src, double* tgt, double alpha_base, int subtract_non_leaf)
{
    auto* h = static_cast<Handle*>(hp);
    return guard([&] {
        const size_t n = h->d->octs.size() * (size_t)h->d->Nb * h->d->Nb * h->d->Nb;
        Field s(src, src + n), t(tgt, tgt + n);
        h->s->apply_if(s, t, alpha_base, subtract_non_leaf != 0);
        std::memcpy(tgt, t.data(), n * sizeof(double));
    });
}

int orc_fmm_apply_ge(void* hp, const double* src, double* tgt, int level, int nlas, double scale, double alpha)
{
    auto* h = static_cast<Handle*>(hp);
    return guard([&] {
        const size_t n = h->d->octs.size() * (size_t)h->d->Nb * h->d->Nb * h->d->Nb;
        Field s(src, src + n), t(tgt, tgt + n);
        h->s->fmm_apply_ge(s, t, level, nlas != 0, scale, alpha);
        std::memcpy(tgt, t.data(), n * sizeof(double));
    });
}

double orc_lgf_ge_get(void* hp, int x, int y, int z, double alpha) { return static_cast<Handle*>(hp)->s->lgf_ge_get(x, y, z, alpha); }

// in/out: arrays of pointers to whole fields (n_oct * Nb^3 each)
int orc_op(void* hp, int op, int n_in, const double* const* in, int n_out, double* const* out, int level,
           double scale)
{
    auto* h = static_cast<Handle*>(hp);
    return guard([&] {
        const size_t n = h->d->octs.size() * (size_t)h->d->Nb * h->d->Nb * h->d->Nb;
        std::vector<Field> fin(n_in), fout(n_out);
        std::vector<const Field*> pin;
        std::vector<Field*> pout;
        for (int i = 0; i < n_in; ++i) fin[i].assign(in[i], in[i] + n), pin.push_back(&fin[i]);
        for (int i = 0; i < n_out; ++i) fout[i].assign(out[i], out[i] + n), pout.push_back(&fout[i]);
        apply_op(*h->d, op, pin, pout, level, scale);
        for (int i = 0; i < n_out; ++i) std::memcpy(out[i], fout[i].data(), n * sizeof(double));
    });
}

int orc_buffer_exchange(void* hp, double* f, int level)
{
    auto* h = static_cast<Handle*>(hp);
    return guard([&] {
        const size_t n = h->d->octs.size() * (size_t)h->d->Nb * h->d->Nb * h->d->Nb;
        Field x(f, f + n);
        buffer_exchange(*h->d, x, level);
        std::memcpy(f, x.data(), n * sizeof(double));
    });
}

// n_steps IF-HERK steps (ifherk.hpp:1078-1200) from time T0: u holds the
// three face-velocity component fields back to back (in/out), p the pressure
// (out).
int orc_ns_step(void* hp, double dt, double Re, double T0, double* u, double* p, int n_steps)
{
    auto* h = static_cast<Handle*>(hp);
    return guard([&] {
        const size_t n = h->d->octs.size() * (size_t)h->d->Nb * h->d->Nb * h->d->Nb;
        Ifherk ns(h->d.get(), h->s.get(), dt, Re);
        ns.T = T0;
        ns.T_last_vel_refresh = h->ns_T_last;
        ns.force_refresh = h->ns_force_refresh;
        for (int k = 0; k < 3; ++k) ns.u.c[k].assign(u + k * n, u + (k + 1) * n);
        for (int st = 0; st < n_steps; ++st) ns.time_step();
        h->ns_T_last = ns.T_last_vel_refresh;
        h->ns_force_refresh = ns.force_refresh;
        for (int k = 0; k < 3; ++k) std::memcpy(u + k * n, ns.u.c[k].data(), n * sizeof(double));
        std::memcpy(p, ns.p.c[0].data(), n * sizeof(double));
    });
}

// IF-HERK steps with an immersed boundary of n_pts points X and a constant
// frame velocity; forces (3 stages x n_pts x 3) gets the stage forces of the
// last step.
int orc_ns_step_ib(void* hp, double dt, double Re, double T0, double* u, double* p, int n_steps, int n_pts,
                   const double* X, const double* frame_vel, double threshold, int max_iter, double* forces)
{
    auto* h = static_cast<Handle*>(hp);
    return guard([&] {
        const size_t n = h->d->octs.size() * (size_t)h->d->Nb * h->d->Nb * h->d->Nb;
        std::vector<std::array<double, 3>> pts(n_pts);
        for (int i = 0; i < n_pts; ++i)
            for (int c = 0; c < 3; ++c) pts[i][c] = X[3 * i + c];
        IbSystem ib(h->d.get(), h->s.get(), pts, Re);
        Ifherk ns(h->d.get(), h->s.get(), dt, Re);
        ns.T = T0;
        ns.T_last_vel_refresh = h->ns_T_last;
        ns.force_refresh = h->ns_force_refresh;
        ns.ib = &ib;
        ns.cg_threshold = threshold;
        ns.cg_max_iter = max_iter;
        for (int k = 0; k < 3; ++k) ns.frame_vel[k] = frame_vel[k];
        for (auto& fp : ns.force_prev) fp.assign(n_pts, {0.0, 0.0, 0.0});
        for (int k = 0; k < 3; ++k) ns.u.c[k].assign(u + k * n, u + (k + 1) * n);
        for (int st = 0; st < n_steps; ++st) ns.time_step();
        h->ns_T_last = ns.T_last_vel_refresh;
        h->ns_force_refresh = ns.force_refresh;
        for (int k = 0; k < 3; ++k) std::memcpy(u + k * n, ns.u.c[k].data(), n * sizeof(double));
        std::memcpy(p, ns.p.c[0].data(), n * sizeof(double));
        for (int sidx = 1; sidx <= 3; ++sidx)
            for (int i = 0; i < n_pts; ++i)
                for (int c = 0; c < 3; ++c) forces[((sidx - 1) * n_pts + i) * 3 + c] = ns.force_prev[sidx][i][c];
    });
}

// IB force solve (linsys.hpp:113-230) for n points X (n x 3): u holds the
// three face-velocity component fields back to back; f (n x 3) is the initial
// guess in and the force out; flags (optional, per octant) gets bit0 is_ib,
// bit1 is_extended_ib; iters gets the CG iteration count.
int orc_ib_solve(void* hp, int n, const double* X, double Re, const double* u, double alpha, double threshold,
                 int max_iter, double* f, int* flags, int* iters)
{
    auto* h = static_cast<Handle*>(hp);
    return guard([&] {
        const size_t N = h->d->octs.size() * (size_t)h->d->Nb * h->d->Nb * h->d->Nb;
        std::vector<std::array<double, 3>> pts(n), force(n);
        for (int i = 0; i < n; ++i)
            for (int c = 0; c < 3; ++c)
            {
                pts[i][c] = X[3 * i + c];
                force[i][c] = f[3 * i + c];
            }
        IbSystem ib(h->d.get(), h->s.get(), pts, Re);
        VField uf;
        uf.mesh = MESH_FACE;
        for (int k = 0; k < 3; ++k) uf.c.emplace_back(u + k * N, u + (k + 1) * N);
        ib.solve(uf, alpha, force, threshold, max_iter);
        for (int i = 0; i < n; ++i)
            for (int c = 0; c < 3; ++c) f[3 * i + c] = force[i][c];
        if (flags)
            for (size_t i = 0; i < h->d->octs.size(); ++i)
                flags[i] = (h->d->octs[i]->ib ? 1 : 0) | (h->d->octs[i]->ext_ib ? 2 : 0);
        if (iters) *iters = ib.iterations;
    });
}

int orc_sphere_points(double dx_base, int ib_level, double ibph, double* X, int cap)
{
    const auto v = sphere_points(dx_base, ib_level, ibph);
    for (int i = 0; i < (int)v.size() && i < cap; ++i)
        for (int c = 0; c < 3; ++c) X[3 * i + c] = v[i][c];
    return (int)v.size();
}

double orc_yang3(double x) { return yang3(x); }

// Single-block linear convolution with the reference's Convolution contract
// (convolution.hpp:225-304): kernel holds P^3 values (P = 2Nb-1, x fastest),
// out (Nb^3) += scale * window[Nb-1, 2Nb-2]^3 of (kernel (*) zero-padded src).
int orc_block_conv(int Nb, const double* src, const double* kernel, double* out, double scale)
{
    return guard([&] {
        const int P = 2 * Nb - 1;
        Fft1d f(P);
        std::vector<cplx> a((size_t)P * P * P, 0.0), b((size_t)P * P * P);
        for (int k = 0; k < Nb; ++k)
            for (int j = 0; j < Nb; ++j)
                for (int i = 0; i < Nb; ++i)
                    a[i + (size_t)P * (j + (size_t)P * k)] = src[i + (size_t)Nb * (j + (size_t)Nb * k)];
        for (size_t i = 0; i < b.size(); ++i) b[i] = kernel[i];
        std::vector<cplx> w(3 * P);
        auto f3 = [&](std::vector<cplx>& x, bool fw) {
            for (int k = 0; k < P; ++k)
                for (int j = 0; j < P; ++j) f.run(&x[(size_t)P * (j + (size_t)P * k)], 1, fw, w.data());
            for (int k = 0; k < P; ++k)
                for (int i = 0; i < P; ++i) f.run(&x[i + (size_t)P * P * k], P, fw, w.data());
            for (int j = 0; j < P; ++j)
                for (int i = 0; i < P; ++i) f.run(&x[i + (size_t)P * j], P * P, fw, w.data());
        };
        f3(a, true);
        f3(b, true);
        const double s = scale / ((double)P * P * P);
        for (size_t i = 0; i < a.size(); ++i) a[i] = a[i] * b[i] * s;
        f3(a, false);
        for (int k = 0; k < Nb; ++k)
            for (int j = 0; j < Nb; ++j)
                for (int i = 0; i < Nb; ++i)
                    out[i + (size_t)Nb * (j + (size_t)Nb * k)] +=
                        a[(i + Nb - 1) + (size_t)P * ((j + Nb - 1) + (size_t)P * (k + Nb - 1))].real();
    });
}

}  // extern "C"
