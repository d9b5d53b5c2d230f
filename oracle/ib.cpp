// ORACLE (test infrastructure): immersed-boundary force solve, restating
//   include/iblgf/domain/ib.hpp:179-210 (sphere points), :652-669
//     (ib_block_overlap), :690-705 (yang3 delta), :70-76 (ddf radius 4.5,
//     safety distance 5 / (Re dx_ib) + 1)
//   domain/decomposition/server.hpp:544-576 (is_ib / is_extended_ib flags),
//     client.hpp:1262-1320 (influence lists and points)
//   operators/operators.hpp:73-170 (clean_ib_region_boundary), :329-517
//     (clean_leaf_correction_boundary), :522-605 (levelDivergence /
//     levelGradient), :841-861 / :996-1013 (ib_projection / ib_smearing, face)
//   solver/linsys/linsys.hpp:113-129 (ib_solve), :170-230 (CG_solve),
//     :263-297 (ET_H_S_E), :299-330 (apply_Schur), :352-376 (smearing),
//     :421-450 (projection).
// Single process: the MPI communication of forces is an identity.
#include <cmath>
#include <stdexcept>

#include "orc.hpp"

namespace orc
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

std::vector<std::array<double, 3>> sphere_points(double dx_base, int ib_level, double ibph)
{
    const double R = 0.5;
    const double dx = dx_base / std::pow(2, ib_level) * ibph;
    const int n = (int)std::floor(M_PI / (dx * dx * 0.86602540378)) + 1;
    const double lambda = (1. + std::sqrt(5)) / 2.0;
    std::vector<std::array<double, 3>> X(n);
    for (int i = 0; i < n; ++i)
    {
        const double x = i + 0.5;
        const double phi = std::acos(1.0 - 2 * x / n);
        const double theta = 2 * M_PI * x / lambda;
        X[i] = {R * std::cos(theta) * std::sin(phi), R * std::sin(theta) * std::sin(phi), R * std::cos(phi)};
    }
    return X;
}

namespace
{
double delta3(double a, double b, double c) { return yang3(a) * yang3(b) * yang3(c); }
}  // namespace

IbSystem::IbSystem(Domain* d_, Solver* s_, const std::vector<std::array<double, 3>>& X_, double Re_)
: d(d_), s(s_), Re(Re_), X(X_)
{
    const int l_max = d->depth - 1;
    ib_level = l_max - d->base_level;
    const double dx_ib = d->dx_base / std::pow(2, ib_level);
    safety_dis = 5.0 / (Re * dx_ib) + 1.0;
    // server.hpp:544-576
    for (Octant* o : d->octs) o->ib = o->ext_ib = false;
    for (size_t i = 0; i < X.size(); ++i)
        for (auto& kv : d->level_maps[l_max])
        {
            Octant* o = kv.second;
            if (!o->has_data) continue;
            if (overlap((int)i, o, 2))
            {
                o->ext_ib = true;
                if (overlap((int)i, o, 1) && o->leaf) o->ib = true;
            }
        }
    fmm_ib_mask_build(*d);
    // client.hpp:1262-1320
    infl.assign(X.size(), {});
    pts.assign(X.size(), {});
    const int e = d->e;
    for (size_t i = 0; i < X.size(); ++i)
    {
        for (auto& kv : d->level_maps[l_max])
        {
            Octant* o = kv.second;
            if (!o->has_data || !o->leaf) continue;
            if (overlap((int)i, o, 1)) infl[i].push_back(o);
        }
        for (Octant* o : infl[i])
        {
            const double sc = std::pow(2, d->refinement_level(o)) / d->dx_base;
            std::vector<std::array<int, 3>> v;
            for (int k = 0; k < e; ++k)
                for (int j = 0; j < e; ++j)
                    for (int a = 0; a < e; ++a)
                    {
                        const int n[3] = {o->bbase[0] + a, o->bbase[1] + j, o->bbase[2] + k};
                        bool in = true;
                        for (int q = 0; q < 3; ++q)
                            if (std::fabs(n[q] - X[i][q] * sc) >= ddf_radius + 1.0) in = false;
                        if (in) v.push_back({a + 1, j + 1, k + 1});
                    }
            pts[i].push_back(v);
        }
    }
    const size_t N = d->octs.size() * (size_t)d->Nb * d->Nb * d->Nb;
    face_aux.mesh = face_aux2.mesh = MESH_FACE;
    face_aux.c.assign(3, Field(N, 0.0));
    face_aux2.c.assign(3, Field(N, 0.0));
    cell_aux2.mesh = MESH_CELL;
    cell_aux2.c.assign(1, Field(N, 0.0));
}

// ib.hpp:652-669: the block, taken to the IB level and grown by the radius of
// radius_level (1: ddf + 5, 2: ddf + safety + 10 cells), contains the point
bool IbSystem::overlap(int i, const Octant* o, int radius_level) const
{
    double r = 0;
    if (radius_level == 2) r = ddf_radius + safety_dis + 10.0;
    else if (radius_level == 1) r = ddf_radius + 5.0;
    const int up = ib_level - d->refinement_level(o);
    const double sc = std::pow(2, up);
    const double factor = std::pow(2, ib_level) / d->dx_base;
    for (int q = 0; q < 3; ++q)
    {
        const double base = o->bbase[q] * sc - r;
        const double ext = d->e * sc + 2 * r;
        const double mx = base + ext - 1;
        if (mx + 1 < X[i][q] * factor || base >= X[i][q] * factor) return false;
    }
    return true;
}

void IbSystem::projection(const VField& u, std::vector<std::array<double, 3>>& f) const
{
    const int Nb = d->Nb;
    const size_t B = (size_t)Nb * Nb * Nb;
    f.assign(X.size(), {0.0, 0.0, 0.0});
    for (size_t i = 0; i < X.size(); ++i)
        for (size_t b = 0; b < infl[i].size(); ++b)
        {
            const Octant* o = infl[i][b];
            const double sc = std::pow(2, d->refinement_level(o)) / d->dx_base;
            for (auto& p : pts[i][b])
            {
                double dist[3];
                for (int q = 0; q < 3; ++q) dist[q] = o->bbase[q] + p[q] - 1 - X[i][q] * sc;
                const size_t at = o->idx * B + p[0] + (size_t)Nb * (p[1] + (size_t)Nb * p[2]);
                for (int c = 0; c < 3; ++c)
                    f[i][c] += u.c[c][at] * delta3(dist[0] + (c == 0 ? 0.0 : 0.5), dist[1] + (c == 1 ? 0.0 : 0.5),
                                                   dist[2] + (c == 2 ? 0.0 : 0.5));
            }
        }
}

void IbSystem::smearing(const std::vector<std::array<double, 3>>& f, VField& u, bool cleaning) const
{
    const int Nb = d->Nb;
    const size_t B = (size_t)Nb * Nb * Nb;
    if (cleaning)
        for (auto& c : u.c) std::fill(c.begin(), c.end(), 0.0);
    for (size_t i = 0; i < X.size(); ++i)
        for (size_t b = 0; b < infl[i].size(); ++b)
        {
            const Octant* o = infl[i][b];
            const double sc = std::pow(2, d->refinement_level(o)) / d->dx_base;
            for (auto& p : pts[i][b])
            {
                double dist[3];
                for (int q = 0; q < 3; ++q) dist[q] = o->bbase[q] + p[q] - 1 - X[i][q] * sc;
                const size_t at = o->idx * B + p[0] + (size_t)Nb * (p[1] + (size_t)Nb * p[2]);
                for (int c = 0; c < 3; ++c)
                    u.c[c][at] += f[i][c] * delta3(dist[0] + (c == 0 ? 0.0 : 0.5), dist[1] + (c == 1 ? 0.0 : 0.5),
                                                   dist[2] + (c == 2 ? 0.0 : 0.5));
            }
        }
}

namespace
{
// zero the outer `width` planes of the face towards face neighbour direction i
void zero_face_planes(double* b, int Nb, int i, int width)
{
    for (int k = 0; k < Nb; ++k)
        for (int j = 0; j < Nb; ++j)
            for (int a = 0; a < Nb; ++a)
            {
                bool z = false;
                if (i == 4) z = k < width;
                else if (i == 10) z = j < width;
                else if (i == 12) z = a < width;
                else if (i == 14) z = a >= Nb - width;
                else if (i == 16) z = j >= Nb - width;
                else if (i == 22) z = k >= Nb - width;
                if (z) b[a + (size_t)Nb * (j + (size_t)Nb * k)] = 0.0;
            }
}
}  // namespace

void IbSystem::clean_ib_region_boundary(VField& f, int l, int width) const
{
    const int Nb = d->Nb;
    const size_t B = (size_t)Nb * Nb * Nb;
    for (auto& kv : d->level_maps[l])
    {
        Octant* o = kv.second;
        for (int i = 0; i < 27; ++i)
        {
            Octant* n = o->neighbor[i];
            if (!n || !n->has_data || !n->ib)
                for (auto& c : f.c) zero_face_planes(&c[o->idx * B], Nb, i, width);
        }
    }
}

void IbSystem::clean_face_boundary(VField& f, int l, bool leaf_only_boundary, int width) const
{
    const int Nb = d->Nb;
    const size_t B = (size_t)Nb * Nb * Nb;
    for (auto& kv : d->level_maps[l])
    {
        Octant* o = kv.second;
        if (leaf_only_boundary && o->correction)
            for (auto& c : f.c) std::fill(&c[o->idx * B], &c[o->idx * B] + B, 0.0);
    }
    if (l != d->base_level) return;
    for (auto& kv : d->level_maps[l])
    {
        Octant* o = kv.second;
        for (int i = 0; i < 27; ++i)
        {
            Octant* n = o->neighbor[i];
            if (!n || !n->has_data || (leaf_only_boundary && n->correction))
                for (auto& c : f.c) zero_face_planes(&c[o->idx * B], Nb, i, width);
        }
    }
}

// apply_Schur<Source, Target>(xIB2IB), linsys.hpp:299-330
void IbSystem::apply_schur(VField& src, VField& tgt)
{
    const int l = d->depth - 1;
    for (auto& c : src.c) buffer_exchange(*d, c, l);
    apply_op(*d, 2, {&src.c[0], &src.c[1], &src.c[2]}, {&cell_aux2.c[0]}, l, 1.0);
    clean_face_boundary(cell_aux2, l, true, 2);
    clean_ib_region_boundary(cell_aux2, l, 2);
    const Field in = cell_aux2.c[0];
    s->apply_lgf(in, cell_aux2.c[0], xIB2IB, true, false);
    apply_op(*d, 1, {&cell_aux2.c[0]}, {&tgt.c[0], &tgt.c[1], &tgt.c[2]}, l, 1.0);
    for (auto& c : tgt.c) buffer_exchange(*d, c, l);
    clean_ib_region_boundary(tgt, l, 2);
}

// ET_H_S_E<face_aux2>, linsys.hpp:263-297
void IbSystem::et_h_s_e(const std::vector<std::array<double, 3>>& fin, std::vector<std::array<double, 3>>& fout,
                        double alpha)
{
    for (auto& c : face_aux.c) std::fill(c.begin(), c.end(), 0.0);
    smearing(fin, face_aux2);
    if (std::fabs(alpha) > 1e-14)
        for (int k = 0; k < 3; ++k)
        {
            int rp[3];
            mesh_relpos(MESH_FACE, k, rp);
            const Field in = face_aux2.c[k];
            s->apply_if(in, face_aux2.c[k], alpha, false, rp, IB2xIB);
        }
    apply_schur(face_aux2, face_aux);
    for (int k = 0; k < 3; ++k)
        for (size_t i = 0; i < face_aux2.c[k].size(); ++i) face_aux2.c[k][i] += face_aux.c[k][i] * -1.0;
    projection(face_aux2, fout);
}

void IbSystem::pressure_correction(const std::vector<std::array<double, 3>>& f, VField& p)
{
    const int l = d->depth - 1;
    for (auto& c : cell_aux2.c) std::fill(c.begin(), c.end(), 0.0);
    smearing(f, face_aux2);
    for (auto& c : face_aux2.c) buffer_exchange(*d, c, l);
    apply_op(*d, 2, {&face_aux2.c[0], &face_aux2.c[1], &face_aux2.c[2]}, {&cell_aux2.c[0]}, l, 1.0);
    clean_face_boundary(cell_aux2, l, true, 2);
    const Field in = cell_aux2.c[0];
    s->apply_lgf(in, cell_aux2.c[0], IB2AMR, true, false);
    for (size_t i = 0; i < p.c[0].size(); ++i) p.c[0][i] += cell_aux2.c[0][i] * -1.0;
}

void IbSystem::solve(const VField& u, double alpha, std::vector<std::array<double, 3>>& f, double threshold,
                     int max_iter)
{
    const size_t n = X.size();
    std::vector<std::array<double, 3>> uc, Ax, r(n), p, Ap;
    projection(u, uc);
    // subtract_boundary_vel: a body at rest in the computational frame
    for (auto& c : face_aux2.c) std::fill(c.begin(), c.end(), 0.0);
    if (f.size() != n) f.assign(n, {0.0, 0.0, 0.0});
    auto dot = [&](const std::vector<std::array<double, 3>>& a, const std::vector<std::array<double, 3>>& b) {
        double s_ = 0.0;
        for (size_t i = 0; i < n; ++i)
            for (int c = 0; c < 3; ++c) s_ += a[i][c] * b[i][c];
        return s_;
    };
    et_h_s_e(f, Ax, alpha);
    for (size_t i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) r[i][c] = uc[i][c] - Ax[i][c];
    p = r;
    double rsold = dot(r, r);
    iterations = 0;
    for (int k = 0; k < max_iter; ++k)
    {
        et_h_s_e(p, Ap, alpha);
        ++iterations;
        const double pAp = dot(p, Ap);
        if (pAp == 0.0) return;
        const double a = rsold / pAp;
        for (size_t i = 0; i < n; ++i)
            for (int c = 0; c < 3; ++c)
            {
                f[i][c] = f[i][c] + p[i][c] * a;
                r[i][c] = r[i][c] + Ap[i][c] * -a;
            }
        const double rsnew = dot(r, r);
        const double f2 = dot(f, f);
        if (std::sqrt(rsnew / f2) < threshold) break;
        for (size_t i = 0; i < n; ++i)
            for (int c = 0; c < 3; ++c) p[i][c] = r[i][c] + p[i][c] * (rsnew / rsold);
        rsold = rsnew;
    }
}
}  // namespace orc
