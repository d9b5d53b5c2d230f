// ORACLE (test infrastructure): FMM masks, Lagrange transfer matrices, block
// FFT convolution, Fmm::apply and PoissonSolver::apply_lgf, restating
//   include/iblgf/fmm/fmm.hpp:54-681 (FmmMaskBuilder), :729-870 (apply),
//     :988-1027 (compute_influence_field), :1029-1165 (add/zero/copy/intrp/antrp),
//     :1167-1195 (fmm_tt)
//   include/iblgf/fmm/fmm_nli.hpp:101-247 (node transfers), :319-374 (matrix)
//   include/iblgf/utilities/convolution.hpp:225-304 (forward add, backward,
//     add_solution), src/utilities/convolution.cpp (pruned r2c / c2r semantics)
//   include/iblgf/lgf/lgf.hpp:78-98,222-262 (spectrum cache, LGF sub-block)
//   include/iblgf/domain/octree/octant.hpp:94-131 (mask indices)
//   include/iblgf/interpolation/cell_center_nli_intrp.hpp:171-238,310-420,
//     557-674,677-787 (cell-centred transfers and source correction)
//   include/iblgf/solver/poisson/poisson.hpp:587-894 (apply_lgf),
//     :921-1013 (copies), :1136-1194 (source_coarsify)
//   include/iblgf/domain/mpi/haloCommunicator.hpp:63-107 (buffer exchange
//     between same-level neighbours on one process).
// Deliberate difference: each source block is transformed once per sweep and
// reused for all its targets; the reference transforms it once per
// (source, target) pair. The transforms are deterministic, so the sums are the
// same. Summation orders otherwise follow the reference.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "orc.hpp"

namespace orc
{
int fmm_mask_idx_gen(int type, int refinement_level, int non_leaf_as_source)
{
    switch (type)
    {
        case STREAM: return 0;
        case IB2xIB: return 1;
        case xIB2IB: return 2;
        case IB2AMR: return refinement_level + 4;
        case AMR2AMR: return refinement_level * 2 + non_leaf_as_source + 15;
        default: throw std::runtime_error("Wrong mask Idx");
    }
}

namespace
{
constexpr int S = 0, T = 1;

void upward_pass(Domain& d, int base_level, int idx)
{
    for (int level = base_level - 1; level >= 0; --level)
    {
        for (auto& kv : d.level_maps[level])
        {
            Octant* o = kv.second;
            o->mask[idx][S] = false;
            for (auto& c : o->child)
                if (c && c->has_data && c->mask[idx][S])
                {
                    o->mask[idx][S] = true;
                    break;
                }
        }
        for (auto& kv : d.level_maps[level])
        {
            Octant* o = kv.second;
            o->mask[idx][T] = false;
            for (auto& c : o->child)
                if (c && c->has_data && c->mask[idx][T])
                {
                    o->mask[idx][T] = true;
                    break;
                }
        }
    }
}

void clean_no_inf(Domain& d, int base_level, int idx)
{
    for (int level = 0; level < base_level; ++level)
    {
        for (auto& kv : d.level_maps[level])
        {
            Octant* o = kv.second;
            if (o->mask[idx][S])
            {
                if (o->parent && o->parent->has_data && o->parent->mask[idx][S]) continue;
                bool has_target = false;
                for (int i = 0; i < o->n_infl; ++i)
                {
                    Octant* n = o->influence[i];
                    if (n && n->has_data && n->mask[idx][T])
                    {
                        has_target = true;
                        break;
                    }
                }
                if (!has_target) o->mask[idx][S] = false;
            }
            if (o->mask[idx][T])
            {
                if (o->parent && o->parent->has_data && o->parent->mask[idx][T]) continue;
                bool has_source = false;
                for (int i = 0; i < o->n_infl; ++i)
                {
                    Octant* n = o->influence[i];
                    if (n && n->has_data && n->mask[idx][S])
                    {
                        has_source = true;
                        break;
                    }
                }
                if (!has_source) o->mask[idx][T] = false;
            }
        }
    }
}

void dry_init(Domain& d, int base_level, bool nlas, int idx, bool subtract)
{
    for (auto& kv : d.level_maps[base_level]) kv.second->mask[idx] = {false, false};
    for (auto& kv : d.level_maps[base_level])
    {
        Octant* o = kv.second;
        if (!o->has_data) continue;
        if (nlas)
        {
            bool corr_parent = false;
            for (auto& c : o->child)
                if (c && c->has_data && c->correction) corr_parent = true;
            if (subtract)
            {
                if (o->leaf || o->correction)
                    o->mask[idx] = {false, corr_parent};
                else
                    o->mask[idx] = {true, true};
            }
            else
            {
                if (o->leaf || o->correction)
                    o->mask[idx] = {true, o->leaf};
                else
                    o->mask[idx] = {false, true};
            }
        }
        else
        {
            if (subtract)
                o->mask[idx] = {true, true};
            else
            {
                if (o->leaf || o->correction)
                    o->mask[idx] = {false, o->leaf};
                else
                    o->mask[idx] = {true, false};
            }
        }
    }
}
}  // namespace

void fmm_lgf_mask_build(Domain& d, bool subtract_non_leaf)
{
    for (int l = d.base_level; l < d.depth; ++l)
    {
        for (int nlas = 0; nlas <= 1; ++nlas)
        {
            const int idx = fmm_mask_idx_gen(AMR2AMR, l - d.base_level, nlas);
            dry_init(d, l, nlas != 0, idx, subtract_non_leaf);
            upward_pass(d, l, idx);
            clean_no_inf(d, l, idx);
        }
    }
}

void fmm_stream_mask_build(Domain& d)
{
    const int idx = fmm_mask_idx_gen(STREAM);
    for (auto& o : d.octs) o->mask[idx] = {false, false};
    for (auto& kv : d.level_maps[d.base_level])
    {
        Octant* o = kv.second;
        if (!o->has_data) continue;
        o->mask[idx] = {!o->correction, true};
    }
    upward_pass(d, d.base_level, idx);
}

void fmm_ib_mask_build(Domain& d)
{
    const int l = d.depth - 1;
    for (int t = IB2xIB; t <= xIB2IB; ++t)
    {
        const int idx = fmm_mask_idx_gen(t);
        for (auto& o : d.octs) o->mask[idx] = {false, false};
        for (auto& kv : d.level_maps[l])
        {
            Octant* o = kv.second;
            if (o->ib) o->mask[idx] = {true, true};
            if (o->ext_ib)
            {
                if (t == IB2xIB) o->mask[idx][T] = true;
                else o->mask[idx][S] = true;
            }
        }
        upward_pass(d, l, idx);
        clean_no_inf(d, l, idx);
    }
    for (int lv = d.depth - 2; lv >= d.base_level; --lv)
        for (auto& kv : d.level_maps[lv])
            for (auto& c : kv.second->child)
                if (c && c->has_data && c->ib) kv.second->ib = true;
    for (int lv = d.depth - 1; lv >= d.base_level; --lv)
    {
        const int idx = fmm_mask_idx_gen(IB2AMR, lv - d.base_level);
        for (auto& o : d.octs) o->mask[idx] = {false, false};
        for (auto& kv : d.level_maps[lv])
        {
            Octant* o = kv.second;
            o->mask[idx][T] = true;
            if (o->ib) o->mask[idx][S] = true;
        }
        upward_pass(d, lv, idx);
    }
}

// fmm_nli.hpp:319-374; mat is Nb x 2Nb with (p, c) at p*2Nb + c
void nli_matrix(int Nb, int pts_cap, double* mat)
{
    std::fill(mat, mat + (size_t)Nb * 2 * Nb, 0.0);
    auto M = [&](int p, int c) -> double& { return mat[(size_t)p * 2 * Nb + c]; };
    for (int c = 1; c < Nb * 2 - 1; ++c)
    {
        const int c_p = c - Nb;
        if (c % 2 == 0)
        {
            M(c / 2, c - 1) = 1.0;
            continue;
        }
        long double sum = 0.0;
        int bl, br;
        if (c_p < -1)
        {
            bl = std::max(0, (c + 1) / 2 - pts_cap / 2);
            br = std::min(Nb, bl + pts_cap);
        }
        else
        {
            br = std::min(Nb, (c + 1) / 2 + pts_cap / 2);
            bl = std::max(0, br - pts_cap);
        }
        for (int p = bl; p < br; ++p)
        {
            long double t = 1.0;
            const int p_p = p * 2 - Nb + 1;
            for (int l = bl; l < br; ++l)
                if (l != p) t /= -(long double)(2 * l - Nb + 1 - p_p);
            t /= (long double)(c_p - p_p + 1);
            M(p, c - 1) = (double)t;
            sum += t;
        }
        for (int p = 0; p < Nb; ++p) M(p, c - 1) /= (double)sum;
    }
    for (int c = Nb * 2 - 1; c > Nb - 1; --c)
        for (int p = 0; p < Nb; ++p) M(p, c) = M(p, c - 2);
}

// cell_center_nli_intrp.hpp:677-787 (relpos 0 identical to nli_matrix)
void cc_matrix(int Nb, int pts_cap, int relpos, double* mat)
{
    if (relpos == 0)
    {
        nli_matrix(Nb, pts_cap, mat);
        return;
    }
    std::fill(mat, mat + (size_t)Nb * 2 * Nb, 0.0);
    auto M = [&](int p, int c) -> double& { return mat[(size_t)p * 2 * Nb + c]; };
    for (int c = 1; c < Nb * 2 - 1; ++c)
    {
        const double c_p = c - Nb + 0.5;
        long double sum = 0.0;
        int bl, br;
        if (c_p < -1)
        {
            bl = std::max(0, (c + 1) / 2 - pts_cap / 2);
            br = std::min(Nb, bl + pts_cap);
        }
        else
        {
            br = std::min(Nb, (c + 1) / 2 + pts_cap / 2);
            bl = std::max(0, br - pts_cap);
        }
        for (int p = bl; p < br; ++p)
        {
            long double t = 1.0;
            const int p_p = p * 2 - Nb + 1;
            for (int l = bl; l < br; ++l)
                if (l != p) t /= -(long double)(2 * l - Nb + 1 - p_p);
            t /= (long double)(c_p - p_p);
            M(p, c - 1) = (double)t;
            sum += t;
        }
        for (int p = 0; p < Nb; ++p) M(p, c - 1) /= (double)sum;
    }
    for (int c = Nb * 2 - 1; c > Nb - 1; --c)
        for (int p = 0; p < Nb; ++p) M(p, c) = M(p, c - 2);
}

namespace
{
// split an Nb x 2Nb matrix into its two Nb x Nb halves, (p, j) at p*Nb + j
void halves(int Nb, const std::vector<double>& full, std::vector<double>* out)
{
    for (int h = 0; h < 2; ++h)
    {
        out[h].assign((size_t)Nb * Nb, 0.0);
        for (int p = 0; p < Nb; ++p)
            for (int j = 0; j < Nb; ++j)
                out[h][(size_t)p * Nb + j] = full[(size_t)p * 2 * Nb + h * Nb + j];
    }
}

// child(i,j,k) (+)= sum Mx(a,i) My(b,j) Mz(c,k) parent(a,b,c); x, then y, then z
void tp_interp(int n, const double* Mx, const double* My, const double* Mz,
               const double* parent, double* child, bool add)
{
    std::vector<double> a2((size_t)n * n * n), a3((size_t)n * n * n);
    auto I = [n](int i, int j, int k) { return (size_t)i + (size_t)n * (j + (size_t)n * k); };
    for (int c = 0; c < n; ++c)
        for (int b = 0; b < n; ++b)
            for (int i = 0; i < n; ++i)
            {
                double s = 0.0;
                for (int a = 0; a < n; ++a) s += parent[I(a, b, c)] * Mx[(size_t)a * n + i];
                a2[I(i, b, c)] = s;
            }
    for (int c = 0; c < n; ++c)
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
            {
                double s = 0.0;
                for (int b = 0; b < n; ++b) s += a2[I(i, b, c)] * My[(size_t)b * n + j];
                a3[I(i, j, c)] = s;
            }
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
            for (int k = 0; k < n; ++k)
            {
                double s = 0.0;
                for (int c = 0; c < n; ++c) s += a3[I(i, j, c)] * Mz[(size_t)c * n + k];
                if (add) child[I(i, j, k)] += s;
                else child[I(i, j, k)] = s;
            }
}

// parent(a,b,c) += sum Mx(a,i) My(b,j) Mz(c,k) child(i,j,k); z, then y, then x
void tp_antrp(int n, const double* Mx, const double* My, const double* Mz,
              const double* child, double* parent)
{
    std::vector<double> a2((size_t)n * n * n), a3((size_t)n * n * n);
    auto I = [n](int i, int j, int k) { return (size_t)i + (size_t)n * (j + (size_t)n * k); };
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            for (int c = 0; c < n; ++c)
            {
                double s = 0.0;
                for (int k = 0; k < n; ++k) s += Mz[(size_t)c * n + k] * child[I(i, j, k)];
                a2[I(i, j, c)] = s;
            }
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < n; ++c)
            for (int b = 0; b < n; ++b)
            {
                double s = 0.0;
                for (int j = 0; j < n; ++j) s += My[(size_t)b * n + j] * a2[I(i, j, c)];
                a3[I(i, b, c)] = s;
            }
    for (int c = 0; c < n; ++c)
        for (int b = 0; b < n; ++b)
            for (int a = 0; a < n; ++a)
            {
                double s = 0.0;
                for (int i = 0; i < n; ++i) s += Mx[(size_t)a * n + i] * a3[I(i, b, c)];
                parent[I(a, b, c)] += s;
            }
}

void fft3(const Fft1d& f, int P, cplx* x, bool forward)
{
    std::vector<cplx> work(3 * P);
    for (int k = 0; k < P; ++k)
        for (int j = 0; j < P; ++j) f.run(x + (size_t)P * (j + (size_t)P * k), 1, forward, work.data());
    for (int k = 0; k < P; ++k)
        for (int i = 0; i < P; ++i) f.run(x + i + (size_t)P * P * k, P, forward, work.data());
    for (int j = 0; j < P; ++j)
        for (int i = 0; i < P; ++i) f.run(x + i + (size_t)P * j, P * P, forward, work.data());
}
}  // namespace

Solver::Solver(Domain* d_, int intrp_order_)
: d(d_)
, Nb(d_->Nb)
, P(2 * d_->Nb - 1)
, intrp_order(intrp_order_)
, fft(2 * d_->Nb - 1)
{
    std::vector<double> full((size_t)Nb * 2 * Nb);
    nli_matrix(Nb, 10, full.data());
    halves(Nb, full, nli_sub);
    std::vector<double> h[2];
    cc_matrix(Nb, intrp_order, 0, full.data());
    halves(Nb, full, h);
    cc_intrp[0] = h[0];
    cc_intrp[1] = h[1];
    cc_matrix(Nb, intrp_order, 1, full.data());
    halves(Nb, full, h);
    cc_intrp[2] = h[0];
    cc_intrp[3] = h[1];
    // coarsify ("simple") matrices, cell_center_nli_intrp.hpp:99-159
    std::vector<double> simple[2];
    for (int r = 0; r < 2; ++r) simple[r].assign((size_t)Nb * (2 * Nb - 2), 0.0);
    auto SM = [&](int r, int i, int c) -> double& { return simple[r][(size_t)i * (2 * Nb - 2) + c]; };
    for (int i = 1; i < Nb - 1; ++i) SM(0, i, i * 2 - 1) = 1.0;
    for (int i = 1; i < Nb - 1; ++i)
    {
        SM(1, i, i * 2 - 1) = 0.5;
        SM(1, i, i * 2) = 0.5;
    }
    for (int s = 0; s < 4; ++s) cc_antrp[s].assign((size_t)Nb * Nb, 0.0);
    for (int p = 0; p < Nb; ++p)
        for (int c = 1; c < Nb - 1; ++c)
        {
            cc_antrp[0][(size_t)p * Nb + c] = SM(0, p, c);
            cc_antrp[1][(size_t)p * Nb + c] = SM(0, p, c + Nb - 2);
            cc_antrp[2][(size_t)p * Nb + c] = SM(1, p, c);
            cc_antrp[3][(size_t)p * Nb + c] = SM(1, p, c + Nb - 2);
        }
}

void Solver::fwd_half(const double* block, std::vector<cplx>& out)
{
    // zero-padded Nb^3 real block in a P^3 box, full complex FFT, keep the
    // half spectrum kx = 0..P/2 laid out [kz][ky][kx]
    const int H = P / 2 + 1;
    std::vector<cplx> x((size_t)P * P * P, 0.0);
    for (int k = 0; k < Nb; ++k)
        for (int j = 0; j < Nb; ++j)
            for (int i = 0; i < Nb; ++i)
                x[i + (size_t)P * (j + (size_t)P * k)] = block[i + (size_t)Nb * (j + (size_t)Nb * k)];
    fft3(fft, P, x.data(), true);
    out.resize((size_t)H * P * P);
    for (int k = 0; k < P; ++k)
        for (int j = 0; j < P; ++j)
            for (int i = 0; i < H; ++i)
                out[i + (size_t)H * (j + (size_t)P * k)] = x[i + (size_t)P * (j + (size_t)P * k)];
}

const std::vector<cplx>& Solver::lgf_spectrum(int ld, int bx, int by, int bz)
{
    const std::array<int, 4> key{ld, bx, by, bz};
    auto it = spectra.find(key);
    if (it != spectra.end()) return it->second;
    // get_subblock: G((base + i) * 2^ld) on the P^3 block, then r2c
    const int step = 1 << ld;
    const int H = P / 2 + 1;
    std::vector<cplx> x((size_t)P * P * P);
    for (int k = 0; k < P; ++k)
        for (int j = 0; j < P; ++j)
            for (int i = 0; i < P; ++i)
                x[i + (size_t)P * (j + (size_t)P * k)] =
                    lgf_get((bx + i) * step, (by + j) * step, (bz + k) * step);
    fft3(fft, P, x.data(), true);
    std::vector<cplx> h((size_t)H * P * P);
    for (int k = 0; k < P; ++k)
        for (int j = 0; j < P; ++j)
            for (int i = 0; i < H; ++i)
                h[i + (size_t)H * (j + (size_t)P * k)] = x[i + (size_t)P * (j + (size_t)P * k)];
    return spectra.emplace(key, std::move(h)).first->second;
}

void Solver::fmm_apply(const Field& src, Field& tgt, int level, bool nlas,
                       double add_with_scale, int fmm_type)
{
    const size_t B = (size_t)Nb * Nb * Nb;
    const int H = P / 2 + 1;
    const size_t NC = (size_t)H * P * P;
    const int rl = level - d->base_level;
    const double dx_level = d->dx_base / std::pow(2.0, rl);
    int idx;
    if (fmm_type == STREAM) idx = fmm_mask_idx_gen(STREAM);
    else if (fmm_type == AMR2AMR) idx = fmm_mask_idx_gen(AMR2AMR, rl, nlas ? 1 : 0);
    else if (fmm_type == IB2xIB || fmm_type == xIB2IB) idx = fmm_mask_idx_gen(fmm_type);
    else if (fmm_type == IB2AMR) idx = fmm_mask_idx_gen(IB2AMR, rl);
    else throw std::runtime_error("oracle: unsupported fmm_type");
    if (fmm_s.size() != d->octs.size() * B) fmm_s.assign(d->octs.size() * B, 0.0);
    if (fmm_t.size() != d->octs.size() * B) fmm_t.assign(d->octs.size() * B, 0.0);
    auto Sm = [&](Octant* o) { return o->mask[idx][S]; };
    auto Tm = [&](Octant* o) { return o->mask[idx][T]; };

    // fmm_init_zero / fmm_init_copy (interior only)
    for (int lv = level; lv >= 0; --lv)
        for (auto& kv : d->level_maps[lv])
        {
            Octant* o = kv.second;
            if (o->has_data && Sm(o)) std::fill(&fmm_s[o->idx * B], &fmm_s[o->idx * B] + B, 0.0);
            if (o->has_data && Tm(o)) std::fill(&fmm_t[o->idx * B], &fmm_t[o->idx * B] + B, 0.0);
        }
    for (auto& kv : d->level_maps[level])
    {
        Octant* o = kv.second;
        if (!(o->has_data && Sm(o))) continue;
        for (int k = 1; k < Nb - 1; ++k)
            for (int j = 1; j < Nb - 1; ++j)
                for (int i = 1; i < Nb - 1; ++i)
                {
                    const size_t c = i + (size_t)Nb * (j + (size_t)Nb * k);
                    fmm_s[o->idx * B + c] = src[o->idx * B + c];
                }
    }
    // targets (sort order of the reference does not change results)
    std::vector<Octant*> targets;
    for (int lv = level; lv >= 0; --lv)
        for (auto& kv : d->level_maps[lv])
            if (kv.second->has_data && Tm(kv.second)) targets.push_back(kv.second);

    // anterpolation
    for (int lv = level - 1; lv >= 0; --lv)
        for (auto& kv : d->level_maps[lv])
        {
            Octant* p = kv.second;
            if (!(p->has_data && Sm(p))) continue;
            for (int c = 0; c < 8; ++c)
            {
                Octant* ch = p->child[c].get();
                if (!ch || !Sm(ch)) continue;
                tp_antrp(Nb, nli_sub[c & 1].data(), nli_sub[(c >> 1) & 1].data(),
                         nli_sub[(c >> 2) & 1].data(), &fmm_s[ch->idx * B], &fmm_s[p->idx * B]);
            }
        }

    // source spectra, once per source block
    std::vector<Octant*> sources;
    for (int lv = level; lv >= 0; --lv)
        for (auto& kv : d->level_maps[lv])
            if (kv.second->has_data && Sm(kv.second)) sources.push_back(kv.second);
    std::map<Octant*, int> sidx;
    for (int i = 0; i < (int)sources.size(); ++i) sidx[sources[i]] = i;
    std::vector<std::vector<cplx>> sspec(sources.size());
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < (int)sources.size(); ++i) fwd_half(&fmm_s[sources[i]->idx * B], sspec[i]);

    // pair lists and spectra (serial cache fill, then parallel over targets)
    struct Pair { int s; const std::vector<cplx>* g; };
    std::vector<std::vector<Pair>> plist(targets.size());
    for (size_t ti = 0; ti < targets.size(); ++ti)
    {
        Octant* t = targets[ti];
        const int ld = level - t->level;
        const bool neighbor = (t->level == level);
        auto add_pair = [&](Octant* s, int lvd) {
            const int bx = t->bbase[0] - s->bbase[0] - (Nb - 1);
            const int by = t->bbase[1] - s->bbase[1] - (Nb - 1);
            const int bz = t->bbase[2] - s->bbase[2] - (Nb - 1);
            plist[ti].push_back({sidx.at(s), &lgf_spectrum(lvd, bx, by, bz)});
        };
        if (neighbor)
            for (int i = 0; i < 27; ++i)
            {
                Octant* n = t->neighbor[i];
                if (n && Sm(n)) add_pair(n, 0);
            }
        for (int i = 0; i < t->n_infl; ++i)
        {
            Octant* n = t->influence[i];
            if (n && Sm(n)) add_pair(n, ld);
        }
    }
    const double scale = dx_level * dx_level / ((double)P * P * P);
#pragma omp parallel for schedule(dynamic)
    for (int ti = 0; ti < (int)targets.size(); ++ti)
    {
        if (plist[ti].empty()) continue;
        Octant* t = targets[ti];
        std::vector<cplx> acc(NC, 0.0);
        for (auto& pr : plist[ti])
        {
            const cplx* g = pr.g->data();
            const cplx* s = sspec[pr.s].data();
            for (size_t f = 0; f < NC; ++f) acc[f] += g[f] * s[f];
        }
        for (size_t f = 0; f < NC; ++f) acc[f] *= scale;
        // c2r: Hermitian extension, complex inverse, real part
        std::vector<cplx> x((size_t)P * P * P);
        for (int k = 0; k < P; ++k)
            for (int j = 0; j < P; ++j)
                for (int i = 0; i < P; ++i)
                {
                    cplx v;
                    if (i < H) v = acc[i + (size_t)H * (j + (size_t)P * k)];
                    else
                    {
                        const int ii = P - i, jj = (P - j) % P, kk = (P - k) % P;
                        v = std::conj(acc[ii + (size_t)H * (jj + (size_t)P * kk)]);
                    }
                    x[i + (size_t)P * (j + (size_t)P * k)] = v;
                }
        fft3(fft, P, x.data(), false);
        double* out = &fmm_t[t->idx * B];
        for (int k = 0; k < Nb; ++k)
            for (int j = 0; j < Nb; ++j)
                for (int i = 0; i < Nb; ++i)
                    out[i + (size_t)Nb * (j + (size_t)Nb * k)] +=
                        x[(i + Nb - 1) + (size_t)P * ((j + Nb - 1) + (size_t)P * (k + Nb - 1))].real();
    }

    // interpolation
    for (int lv = 1; lv < level; ++lv)
        for (auto& kv : d->level_maps[lv])
        {
            Octant* p = kv.second;
            if (!(p->has_data && Tm(p))) continue;
            for (int c = 0; c < 8; ++c)
            {
                Octant* ch = p->child[c].get();
                if (!ch || !Tm(ch) || !ch->has_data) continue;
                tp_interp(Nb, nli_sub[c & 1].data(), nli_sub[(c >> 1) & 1].data(),
                          nli_sub[(c >> 2) & 1].data(), &fmm_t[p->idx * B], &fmm_t[ch->idx * B], true);
            }
        }
    // fmm_add_equal
    for (auto& kv : d->level_maps[level])
    {
        Octant* o = kv.second;
        if (!(o->has_data && Tm(o))) continue;
        for (size_t c = 0; c < B; ++c) tgt[o->idx * B + c] += fmm_t[o->idx * B + c] * add_with_scale;
    }
}

void Solver::apply_lgf(const Field& src, Field& tgt, int fmm_type, bool use_correction,
                       bool subtract_non_leaf)
{
    if (fmm_type != AMR2AMR && fmm_type != STREAM && fmm_type != xIB2IB && fmm_type != IB2xIB &&
        fmm_type != IB2AMR)
        throw std::runtime_error("oracle: unsupported fmm_type");
    const size_t B = (size_t)Nb * Nb * Nb;
    const size_t N = d->octs.size() * B;
    Field source_tmp(N, 0.0), target_tmp(N, 0.0), correction_tmp(N, 0.0);
    auto blk = [&](Field& f, Octant* o) { return &f[o->idx * B]; };
    if (fmm_type == STREAM)
    {
        // poisson.hpp:612-614 (copy_level, interior only), l = base level only,
        // one sweep with the stream mask (:749-752), leaves copied (:761-781)
        for (auto& kv : d->level_maps[d->base_level])
        {
            Octant* o = kv.second;
            for (int k = 1; k < Nb - 1; ++k)
                for (int j = 1; j < Nb - 1; ++j)
                    for (int i = 1; i < Nb - 1; ++i)
                    {
                        const size_t c = i + (size_t)Nb * (j + (size_t)Nb * k);
                        source_tmp[o->idx * B + c] = src[o->idx * B + c];
                    }
        }
        if (!subtract_non_leaf)
        {
            fmm_apply(source_tmp, target_tmp, d->base_level, false, 1.0, STREAM);
            for (auto& kv : d->level_maps[d->base_level])
            {
                Octant* o = kv.second;
                if (o->leaf) std::copy(blk(target_tmp, o), blk(target_tmp, o) + B, &tgt[o->idx * B]);
            }
        }
        return;
    }
    if (fmm_type == xIB2IB || fmm_type == IB2xIB)
    {
        // poisson.hpp:615-616, 648-650, 702-745: finest level only, interior
        // copy, one sweep with the IB mask, leaves of that level assigned
        const int l = d->depth - 1;
        copy_level_interior(src, source_tmp, l);
        if (!subtract_non_leaf)
        {
            fmm_apply(source_tmp, target_tmp, l, false, 1.0, fmm_type);
            for (auto& kv : d->level_maps[l])
            {
                Octant* o = kv.second;
                if (o->leaf) std::copy(blk(target_tmp, o), blk(target_tmp, o) + B, &tgt[o->idx * B]);
            }
        }
        return;
    }
    if (fmm_type == IB2AMR)
    {
        // poisson.hpp:617-618, 632-634, 702-745: finest-level interior copy,
        // coarsified (cell mesh), one sweep per level with the IB2AMR mask,
        // leaves assigned; no source correction
        copy_level_interior(src, source_tmp, d->depth - 1);
        coarsify_all(source_tmp);
        for (int l = d->base_level; l < d->depth && !subtract_non_leaf; ++l)
        {
            fmm_apply(source_tmp, target_tmp, l, false, 1.0, IB2AMR);
            for (auto& kv : d->level_maps[l])
            {
                Octant* o = kv.second;
                if (o->leaf) std::copy(blk(target_tmp, o), blk(target_tmp, o) + B, &tgt[o->idx * B]);
            }
        }
        return;
    }
    // copy_leaf (with buffer)
    for (Octant* o : d->octs)
        if (o->leaf) std::copy(&src[o->idx * B], &src[o->idx * B] + B, blk(source_tmp, o));
    // source_coarsify: cell-centred 2-point average per axis
    for (int ls = d->depth - 2; ls >= d->base_level; --ls)
        for (auto& kv : d->level_maps[ls])
        {
            Octant* p = kv.second;
            for (int c = 0; c < 8; ++c)
            {
                Octant* ch = p->child[c].get();
                if (!ch || !ch->has_data) continue;
                tp_antrp(Nb, cc_antrp[2 + (c & 1)].data(), cc_antrp[2 + ((c >> 1) & 1)].data(),
                         cc_antrp[2 + ((c >> 2) & 1)].data(), blk(source_tmp, ch), blk(source_tmp, p));
            }
        }
    for (int l = d->base_level; l < d->depth; ++l)
    {
        if (!subtract_non_leaf)
        {
            fmm_apply(source_tmp, target_tmp, l, true, 1.0, AMR2AMR);
            for (auto& kv : d->level_maps[l])
            {
                Octant* p = kv.second;
                for (int c = 0; c < 8; ++c)
                {
                    Octant* ch = p->child[c].get();
                    if (!ch || !ch->has_data) continue;
                    tp_interp(Nb, cc_intrp[2 + (c & 1)].data(), cc_intrp[2 + ((c >> 1) & 1)].data(),
                              cc_intrp[2 + ((c >> 2) & 1)].data(), blk(target_tmp, p),
                              blk(target_tmp, ch), false);
                }
            }
            fmm_apply(source_tmp, target_tmp, l, false, 1.0, AMR2AMR);
            for (auto& kv : d->level_maps[l])
            {
                Octant* o = kv.second;
                if (o->leaf) std::copy(blk(target_tmp, o), blk(target_tmp, o) + B, &tgt[o->idx * B]);
            }
        }
        if (!use_correction || l == d->depth - 1) continue;
        // buffer exchange of source_tmp at level l
        for (auto& kv : d->level_maps[l])
        {
            Octant* o = kv.second;
            double* dst = blk(source_tmp, o);
            for (int ni = 0; ni < 27; ++ni)
            {
                Octant* n = o->neighbor[ni];
                if (!n || !n->has_data || n == o) continue;
                const double* sp = blk(source_tmp, n);
                // overlap of n's interior with o's real block, in global cells
                for (int k = 0; k < Nb; ++k)
                    for (int j = 0; j < Nb; ++j)
                        for (int i = 0; i < Nb; ++i)
                        {
                            const int gx = o->bbase[0] - 1 + i, gy = o->bbase[1] - 1 + j,
                                      gz = o->bbase[2] - 1 + k;
                            const int li = gx - n->bbase[0], lj = gy - n->bbase[1], lk = gz - n->bbase[2];
                            if (li < 0 || lj < 0 || lk < 0 || li >= d->e || lj >= d->e || lk >= d->e)
                                continue;
                            dst[i + (size_t)Nb * (j + (size_t)Nb * k)] =
                                sp[(li + 1) + (size_t)Nb * ((lj + 1) + (size_t)Nb * (lk + 1))];
                        }
            }
        }
        for (auto& kv : d->level_maps[l])
        {
            Octant* p = kv.second;
            for (int c = 0; c < 8; ++c)
            {
                Octant* ch = p->child[c].get();
                if (!ch || !ch->has_data || !ch->correction) continue;
                tp_interp(Nb, cc_intrp[2 + (c & 1)].data(), cc_intrp[2 + ((c >> 1) & 1)].data(),
                          cc_intrp[2 + ((c >> 2) & 1)].data(), blk(source_tmp, p),
                          blk(correction_tmp, ch), false);
            }
        }
        for (auto& kv : d->level_maps[l])
        {
            Octant* p = kv.second;
            const double dx = d->dx_base / std::pow(2.0, l - d->base_level) / 2.0;
            const double r = 1.0 / (dx * dx);
            for (int c = 0; c < 8; ++c)
            {
                Octant* ch = p->child[c].get();
                if (!ch || !ch->has_data) continue;
                const double* tt = blk(target_tmp, ch);
                double* cc = blk(correction_tmp, ch);
                auto I = [&](int i, int j, int k) { return i + (size_t)Nb * (j + (size_t)Nb * k); };
                for (int i = 1; i < Nb - 1; ++i)
                    for (int j = 1; j < Nb - 1; ++j)
                        for (int k = 1; k < Nb - 1; ++k)
                        {
                            double& v = cc[I(i, j, k)];
                            v += 6.0 * tt[I(i, j, k)] * r;
                            v -= tt[I(i, j, k - 1)] * r;
                            v -= tt[I(i, j, k + 1)] * r;
                            v -= tt[I(i, j - 1, k)] * r;
                            v -= tt[I(i, j + 1, k)] * r;
                            v -= tt[I(i + 1, j, k)] * r;
                            v -= tt[I(i - 1, j, k)] * r;
                            v += 0.0 * tt[I(i, j, k)];
                        }
            }
        }
        for (auto& kv : d->level_maps[l + 1])
        {
            Octant* o = kv.second;
            for (size_t c = 0; c < B; ++c) source_tmp[o->idx * B + c] += correction_tmp[o->idx * B + c];
        }
    }
}

}  // namespace orc

// ---------------------------------------------------------------------------
// Integrating-factor kernel LGF_GE (include/iblgf/lgf/lgf_ge.hpp:33-190):
// E(n; alpha) = e^{-6 alpha} I_n1(2 alpha) I_n2(2 alpha) I_n3(2 alpha)
//             = prod_i e^{-2 alpha} I_ni(2 alpha), neighbour-only, alpha scaled
// by 4^level_diff (change_level_impl :81-84); the FMM takes the short branch
// of Fmm::apply (fmm.hpp:754-770) with scale 1 (no dx^2).
namespace orc
{
double Solver::lgf_ge_get(int x, int y, int z, double alpha)
{
    const int nmax = 4 * Nb + 8;
    if (alpha != ge_alpha || (int)ge_f.size() < nmax + 1)
    {
        ge_f.assign(nmax + 1, 0.0);
        bessel_ie_all(2.0 * alpha, nmax, ge_f.data());
        ge_alpha = alpha;
    }
    x = std::abs(x);
    y = std::abs(y);
    z = std::abs(z);
    if (x > nmax || y > nmax || z > nmax) throw std::runtime_error("LGF_GE offset out of range");
    return ge_f[x] * ge_f[y] * ge_f[z];
}

const std::vector<cplx>& Solver::lgf_ge_spectrum(double alpha, int bx, int by, int bz)
{
    const auto key = std::make_tuple(alpha, bx, by, bz);
    auto it = spectra_ge.find(key);
    if (it != spectra_ge.end()) return it->second;
    const int H = P / 2 + 1;
    std::vector<cplx> x((size_t)P * P * P);
    for (int k = 0; k < P; ++k)
        for (int j = 0; j < P; ++j)
            for (int i = 0; i < P; ++i)
                x[i + (size_t)P * (j + (size_t)P * k)] = lgf_ge_get(bx + i, by + j, bz + k, alpha);
    fft3(fft, P, x.data(), true);
    std::vector<cplx> h((size_t)H * P * P);
    for (int k = 0; k < P; ++k)
        for (int j = 0; j < P; ++j)
            for (int i = 0; i < H; ++i)
                h[i + (size_t)H * (j + (size_t)P * k)] = x[i + (size_t)P * (j + (size_t)P * k)];
    return spectra_ge.emplace(key, std::move(h)).first->second;
}

void Solver::fmm_apply_ge(const Field& src, Field& tgt, int level, bool nlas, double add_with_scale,
                          double alpha, int fmm_type)
{
    const size_t B = (size_t)Nb * Nb * Nb;
    const int H = P / 2 + 1;
    const size_t NC = (size_t)H * P * P;
    const int rl = level - d->base_level;
    const int idx = fmm_type == AMR2AMR ? fmm_mask_idx_gen(AMR2AMR, rl, nlas ? 1 : 0) : fmm_mask_idx_gen(fmm_type, rl);
    if (fmm_s.size() != d->octs.size() * B) fmm_s.assign(d->octs.size() * B, 0.0);
    if (fmm_t.size() != d->octs.size() * B) fmm_t.assign(d->octs.size() * B, 0.0);
    auto Sm = [&](Octant* o) { return o->mask[idx][0]; };
    auto Tm = [&](Octant* o) { return o->mask[idx][1]; };
    for (int lv = level; lv >= 0; --lv)
        for (auto& kv : d->level_maps[lv])
        {
            Octant* o = kv.second;
            if (o->has_data && Sm(o)) std::fill(&fmm_s[o->idx * B], &fmm_s[o->idx * B] + B, 0.0);
            if (o->has_data && Tm(o)) std::fill(&fmm_t[o->idx * B], &fmm_t[o->idx * B] + B, 0.0);
        }
    for (auto& kv : d->level_maps[level])
    {
        Octant* o = kv.second;
        if (!(o->has_data && Sm(o))) continue;
        for (int k = 1; k < Nb - 1; ++k)
            for (int j = 1; j < Nb - 1; ++j)
                for (int i = 1; i < Nb - 1; ++i)
                {
                    const size_t c = i + (size_t)Nb * (j + (size_t)Nb * k);
                    fmm_s[o->idx * B + c] = src[o->idx * B + c];
                }
    }
    std::vector<Octant*> targets, sources;
    for (auto& kv : d->level_maps[level])
    {
        if (kv.second->has_data && Tm(kv.second)) targets.push_back(kv.second);
        if (kv.second->has_data && Sm(kv.second)) sources.push_back(kv.second);
    }
    std::map<Octant*, int> sidx;
    for (int i = 0; i < (int)sources.size(); ++i) sidx[sources[i]] = i;
    std::vector<std::vector<cplx>> sspec(sources.size());
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < (int)sources.size(); ++i) fwd_half(&fmm_s[sources[i]->idx * B], sspec[i]);
    struct Pair { int s; const std::vector<cplx>* g; };
    std::vector<std::vector<Pair>> plist(targets.size());
    for (size_t ti = 0; ti < targets.size(); ++ti)
    {
        Octant* t = targets[ti];
        for (int i = 0; i < 27; ++i)
        {
            Octant* n = t->neighbor[i];
            if (!n || !Sm(n)) continue;
            plist[ti].push_back({sidx.at(n), &lgf_ge_spectrum(alpha, t->bbase[0] - n->bbase[0] - (Nb - 1),
                                                              t->bbase[1] - n->bbase[1] - (Nb - 1),
                                                              t->bbase[2] - n->bbase[2] - (Nb - 1))});
        }
    }
    const double scale = 1.0 / ((double)P * P * P);
#pragma omp parallel for schedule(dynamic)
    for (int ti = 0; ti < (int)targets.size(); ++ti)
    {
        if (plist[ti].empty()) continue;
        std::vector<cplx> acc(NC, 0.0);
        for (auto& pr : plist[ti])
        {
            const cplx* g = pr.g->data();
            const cplx* s = sspec[pr.s].data();
            for (size_t f = 0; f < NC; ++f) acc[f] += g[f] * s[f];
        }
        for (size_t f = 0; f < NC; ++f) acc[f] *= scale;
        std::vector<cplx> x((size_t)P * P * P);
        for (int k = 0; k < P; ++k)
            for (int j = 0; j < P; ++j)
                for (int i = 0; i < P; ++i)
                {
                    cplx v;
                    if (i < H) v = acc[i + (size_t)H * (j + (size_t)P * k)];
                    else v = std::conj(acc[(P - i) + (size_t)H * ((P - j) % P + (size_t)P * ((P - k) % P))]);
                    x[i + (size_t)P * (j + (size_t)P * k)] = v;
                }
        fft3(fft, P, x.data(), false);
        double* out = &fmm_t[targets[ti]->idx * B];
        for (int k = 0; k < Nb; ++k)
            for (int j = 0; j < Nb; ++j)
                for (int i = 0; i < Nb; ++i)
                    out[i + (size_t)Nb * (j + (size_t)Nb * k)] +=
                        x[(i + Nb - 1) + (size_t)P * ((j + Nb - 1) + (size_t)P * (k + Nb - 1))].real();
    }
    for (auto& kv : d->level_maps[level])
    {
        Octant* o = kv.second;
        if (!(o->has_data && Tm(o))) continue;
        for (size_t c = 0; c < B; ++c) tgt[o->idx * B + c] += fmm_t[o->idx * B + c] * add_with_scale;
    }
}

void Solver::coarsify_all(Field& f, const int* rp)
{
    const size_t B = (size_t)Nb * Nb * Nb;
    static const int cell[3] = {1, 1, 1};
    if (!rp) rp = cell;
    for (int ls = d->depth - 2; ls >= d->base_level; --ls)
        for (auto& kv : d->level_maps[ls])
        {
            Octant* p = kv.second;
            for (int c = 0; c < 8; ++c)
            {
                Octant* ch = p->child[c].get();
                if (!ch || !ch->has_data) continue;
                tp_antrp(Nb, cc_antrp[2 * rp[0] + (c & 1)].data(), cc_antrp[2 * rp[1] + ((c >> 1) & 1)].data(),
                         cc_antrp[2 * rp[2] + ((c >> 2) & 1)].data(), &f[ch->idx * B], &f[p->idx * B]);
            }
        }
}

void Solver::cc_intrp_level(Field& from, Field& to, int level, bool correction_only, const int* rp)
{
    const size_t B = (size_t)Nb * Nb * Nb;
    static const int cell[3] = {1, 1, 1};
    if (!rp) rp = cell;
    for (auto& kv : d->level_maps[level])
    {
        Octant* p = kv.second;
        for (int c = 0; c < 8; ++c)
        {
            Octant* ch = p->child[c].get();
            if (!ch || !ch->has_data) continue;
            if (correction_only && !ch->correction) continue;
            tp_interp(Nb, cc_intrp[2 * rp[0] + (c & 1)].data(), cc_intrp[2 * rp[1] + ((c >> 1) & 1)].data(),
                      cc_intrp[2 * rp[2] + ((c >> 2) & 1)].data(), &from[p->idx * B], &to[ch->idx * B], false);
        }
    }
}

void Solver::cc_intrp_child(Field& f, Octant* p, int c, const int* rp)
{
    const size_t B = (size_t)Nb * Nb * Nb;
    Octant* ch = p->child[c].get();
    tp_interp(Nb, cc_intrp[2 * rp[0] + (c & 1)].data(), cc_intrp[2 * rp[1] + ((c >> 1) & 1)].data(),
              cc_intrp[2 * rp[2] + ((c >> 2) & 1)].data(), &f[p->idx * B], &f[ch->idx * B], false);
}

// PoissonSolver::apply_if (poisson.hpp:436-494) for AMR2AMR; rp: relative
// positions of the field's mesh object (cell {1,1,1} when null)
void Solver::apply_if(const Field& src, Field& tgt, double alpha_base, bool subtract_non_leaf, const int* rp,
                      int fmm_type)
{
    const size_t B = (size_t)Nb * Nb * Nb;
    const size_t N = d->octs.size() * B;
    Field source_tmp(N, 0.0), target_tmp(N, 0.0);
    if (fmm_type == AMR2AMR)
    {
        for (Octant* o : d->octs)
            if (o->leaf) std::copy(&src[o->idx * B], &src[o->idx * B] + B, &source_tmp[o->idx * B]);
        coarsify_all(source_tmp, rp);
        // intrp_to_correction_buffer (poisson.hpp:1015-1069)
        for (int l = d->depth - 2; l >= d->base_level; --l)
        {
            buffer_exchange(*d, source_tmp, l);
            cc_intrp_level(source_tmp, source_tmp, l, true, rp);
        }
    }
    else if (fmm_type == IB2xIB)
        copy_level_interior(src, source_tmp, d->depth - 1);
    else
        throw std::runtime_error("oracle: apply_if supports AMR2AMR and IB2xIB");
    const int l_min = fmm_type == IB2xIB ? d->depth - 1 : d->base_level;
    for (int l = l_min; l < d->depth; ++l)
    {
        const double alpha = alpha_base * std::pow(4.0, l - d->base_level);
        if (fmm_type == AMR2AMR) fmm_apply_ge(source_tmp, target_tmp, l, false, 1.0, alpha, fmm_type);
        if (!subtract_non_leaf) fmm_apply_ge(source_tmp, target_tmp, l, true, 1.0, alpha, fmm_type);
        for (auto& kv : d->level_maps[l])
        {
            Octant* o = kv.second;
            std::copy(&target_tmp[o->idx * B], &target_tmp[o->idx * B] + B, &tgt[o->idx * B]);
        }
    }
}

// copy_level(l, with_buffer = false): interior nodes of every block of level l
void Solver::copy_level_interior(const Field& src, Field& dst, int l) const
{
    for (auto& kv : d->level_maps[l])
    {
        Octant* o = kv.second;
        const size_t B = (size_t)Nb * Nb * Nb;
        for (int k = 1; k < Nb - 1; ++k)
            for (int j = 1; j < Nb - 1; ++j)
                for (int i = 1; i < Nb - 1; ++i)
                {
                    const size_t c = i + (size_t)Nb * (j + (size_t)Nb * k);
                    dst[o->idx * B + c] = src[o->idx * B + c];
                }
    }
}
}  // namespace orc
