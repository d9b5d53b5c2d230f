// ORACLE (test infrastructure): one IF-HERK time step of the incompressible
// Navier-Stokes solver, restating
//   include/iblgf/solver/time_integration/ifherk.hpp
//     :164-173   alpha_k = (c_{k+1} - c_k) dt / (Re dx_base^2)
//     :992-1015  up_and_down / up / down_to_correction
//     :1078-1200 time_step (3 stages, a = {1/3, -1, 2, 0, 3/4, 1/4},
//                c = {0, 1/3, 1, 1}, :2010-2011)
//     :1309-1352 clean, :1355-1405 clean_leaf_correction_boundary
//     :1451-1517 lin_sys_with_ib_solve
//     :1638-1692 nonlinear, :1738-1763 divergence, :1766-1795 gradient
//     :1878-1960 add / copy
//   include/iblgf/operators/operators.hpp:653-760 smooth2zero
//   include/iblgf/interpolation/cell_center_nli_intrp.hpp:349-365 relative
//     positions of cell / face / edge components.
//     :1093-1111 velocity refresh once (T - T_last_refresh) 3.3 / (Re dx^2) > 7:
//                pad_velocity (:1522-1573, refresh_correction_only) and
//                adapt_corr_time_step (:1206-1303)
// Scope: optional immersed boundary, constant frame velocity, no adaptation,
// no body force.
#include <cmath>
#include <stdexcept>

#include "orc.hpp"

namespace orc
{
void mesh_relpos(int mesh, int comp, int rp[3])
{
    for (int a = 0; a < 3; ++a) rp[a] = 1;
    if (mesh == MESH_FACE) rp[comp] = 0;
    else if (mesh == MESH_EDGE)
    {
        for (int a = 0; a < 3; ++a) rp[a] = 0;
        rp[comp] = 1;
    }
}

Ifherk::Ifherk(Domain* d_, Solver* s_, double dt_, double Re_) : d(d_), s(s_), dt(dt_), Re(Re_)
{
    const size_t N = d->octs.size() * (size_t)d->Nb * d->Nb * d->Nb;
    auto mk = [N](VField& f, int mesh, int n) {
        f.mesh = mesh;
        f.c.assign(n, Field(N, 0.0));
    };
    mk(u, MESH_FACE, 3);
    mk(p, MESH_CELL, 1);
    mk(q_i, MESH_FACE, 3);
    mk(g_i, MESH_FACE, 3);
    mk(d_i, MESH_CELL, 1);
    mk(r_i, MESH_FACE, 3);
    mk(u_i, MESH_FACE, 3);
    mk(w_1, MESH_FACE, 3);
    mk(w_2, MESH_FACE, 3);
    mk(cell_aux, MESH_CELL, 1);
    mk(face_aux, MESH_FACE, 3);
    mk(edge_aux, MESH_EDGE, 3);
    mk(stream_f, MESH_EDGE, 3);
    const double tmp = Re * d->dx_base * d->dx_base / dt;
    for (int k = 0; k < 3; ++k) alpha[k] = (c[k + 1] - c[k]) / tmp;
}

double Ifherk::coeff_a(int i, int j) const { return a[i * (i - 1) / 2 + j - 1]; }

void Ifherk::clean(VField& f, bool non_leaf_only)
{
    const int Nb = d->Nb;
    const size_t B = (size_t)Nb * Nb * Nb;
    for (Octant* o : d->octs)
        for (auto& comp : f.c)
        {
            double* b = &comp[o->idx * B];
            if (non_leaf_only && o->leaf)
            {
                for (int k = 0; k < Nb; ++k)
                    for (int j = 0; j < Nb; ++j)
                        for (int i = 0; i < Nb; ++i)
                            if (i == 0 || j == 0 || k == 0 || i == Nb - 1 || j == Nb - 1 || k == Nb - 1)
                                b[i + (size_t)Nb * (j + (size_t)Nb * k)] = 0.0;
            }
            else
                std::fill(b, b + B, 0.0);
        }
}

void Ifherk::up(VField& f)
{
    for (size_t k = 0; k < f.c.size(); ++k)
    {
        int rp[3];
        mesh_relpos(f.mesh, (int)k, rp);
        s->coarsify_all(f.c[k], rp);
    }
}

void Ifherk::down_to_correction(VField& f)
{
    for (size_t k = 0; k < f.c.size(); ++k)
    {
        int rp[3];
        mesh_relpos(f.mesh, (int)k, rp);
        for (int l = d->depth - 2; l >= d->base_level; --l)
        {
            buffer_exchange(*d, f.c[k], l);
            s->cc_intrp_level(f.c[k], f.c[k], l, true, rp);
        }
    }
}

void Ifherk::up_and_down(VField& f)
{
    clean(f, true);
    up(f);
    down_to_correction(f);
}

void Ifherk::smooth2zero(VField& f, Octant* o, int ngb)
{
    const int Nb = d->Nb;
    const size_t B = (size_t)Nb * Nb * Nb;
    const int x = ngb % 3, y = (ngb / 3) % 3, z = ngb / 9;
    const double fac = 10.0, shift = 0.2;
    const double cst = 1.0 - (0.5 + 0.5 * std::tanh(fac * (1.0 - shift)));
    auto fn = [&](double v) { return (0.5 + 0.5 * std::tanh(fac * (v - shift))) + cst; };
    for (auto& comp : f.c)
    {
        double* b = &comp[o->idx * B];
        for (int k = 0; k < Nb; ++k)
            for (int j = 0; j < Nb; ++j)
                for (int i = 0; i < Nb; ++i)
                {
                    // local_pct over the block with its buffer (node.hpp:121-124)
                    const double px = (double)i / (Nb - 1), py = (double)j / (Nb - 1), pz = (double)k / (Nb - 1);
                    double sq = 0.0;
                    int cnt = 0;
                    if (z == 0) sq = std::max(sq, fn(pz)), ++cnt;
                    else if (z == 2) sq = std::max(sq, fn(1.0 - pz)), ++cnt;
                    if (y == 0) sq = std::max(sq, fn(py)), ++cnt;
                    else if (y == 2) sq = std::max(sq, fn(1.0 - py)), ++cnt;
                    if (x == 0) sq = std::max(sq, fn(px)), ++cnt;
                    else if (x == 2) sq = std::max(sq, fn(1.0 - px)), ++cnt;
                    if (cnt > 0) b[i + (size_t)Nb * (j + (size_t)Nb * k)] *= sq;
                }
    }
}

void Ifherk::clean_leaf_correction_boundary(VField& f, int l, bool leaf_only_boundary)
{
    const size_t B = (size_t)d->Nb * d->Nb * d->Nb;
    for (auto& kv : d->level_maps[l])
    {
        Octant* o = kv.second;
        if (leaf_only_boundary && (o->correction || o->old_correction))
            for (auto& comp : f.c) std::fill(&comp[o->idx * B], &comp[o->idx * B] + B, 0.0);
    }
    if (l != d->base_level) return;
    for (auto& kv : d->level_maps[l])
    {
        Octant* o = kv.second;
        for (int i = 0; i < 27; ++i)
        {
            Octant* n = o->neighbor[i];
            if (!n || !n->has_data || (leaf_only_boundary && (n->correction || n->old_correction)))
                // the reference calls smooth2zero (which scales every
                // component) once per component of the field
                for (size_t rep = 0; rep < f.c.size(); ++rep) smooth2zero(f, o, i);
        }
    }
}

void Ifherk::op_level(int op, const std::vector<const Field*>& in, const std::vector<Field*>& out, int l,
                      double scale)
{
    apply_op(*d, op, in, out, l, scale);
}

void Ifherk::exchange(VField& f, int l)
{
    for (auto& comp : f.c) buffer_exchange(*d, comp, l);
}

void Ifherk::copy(const VField& from, VField& to, double scale)
{
    for (size_t k = 0; k < from.c.size(); ++k)
        for (size_t i = 0; i < from.c[k].size(); ++i) to.c[k][i] = from.c[k][i] * scale;
}

void Ifherk::add(const VField& from, VField& to, double scale)
{
    for (size_t k = 0; k < from.c.size(); ++k)
        for (size_t i = 0; i < from.c[k].size(); ++i) to.c[k][i] += from.c[k][i] * scale;
}

void Ifherk::nonlinear(VField& src, VField& tgt, double scale)
{
    clean(edge_aux, false);
    clean(tgt, false);
    clean(face_aux, false);
    for (int l = d->base_level; l < d->depth; ++l)
    {
        exchange(src, l);
        op_level(3, {&src.c[0], &src.c[1], &src.c[2]}, {&edge_aux.c[0], &edge_aux.c[1], &edge_aux.c[2]}, l, 1.0);
    }
    copy(src, face_aux, 1.0);
    // add_field_expression(frame_vel, -1): a constant frame velocity
    for (int k = 0; k < 3; ++k)
        if (frame_vel[k] != 0.0)
            for (double& v : face_aux.c[k]) v += frame_vel[k] * -1.0;
    for (int l = d->base_level; l < d->depth; ++l)
    {
        exchange(edge_aux, l);
        clean_leaf_correction_boundary(edge_aux, l, false);
        op_level(5,
                 {&face_aux.c[0], &face_aux.c[1], &face_aux.c[2], &edge_aux.c[0], &edge_aux.c[1], &edge_aux.c[2]},
                 {&tgt.c[0], &tgt.c[1], &tgt.c[2]}, l, 1.0);
    }
    for (auto& comp : tgt.c)
        for (double& v : comp) v *= scale;
}

void Ifherk::divergence(VField& src, VField& tgt)
{
    up_and_down(src);
    for (int l = d->base_level; l < d->depth; ++l)
    {
        exchange(src, l);
        op_level(2, {&src.c[0], &src.c[1], &src.c[2]}, {&tgt.c[0]}, l, 1.0);
        clean_leaf_correction_boundary(tgt, l, true);
    }
}

void Ifherk::gradient(VField& src, VField& tgt)
{
    clean(tgt, false);
    for (int l = d->base_level; l < d->depth; ++l)
    {
        op_level(1, {&src.c[0]}, {&tgt.c[0], &tgt.c[1], &tgt.c[2]}, l, 1.0);
        exchange(tgt, l);
    }
}

void Ifherk::apply_if(const VField& src, VField& tgt, double alpha_base)
{
    for (size_t k = 0; k < src.c.size(); ++k)
    {
        int rp[3];
        mesh_relpos(src.mesh, (int)k, rp);
        const Field in = src.c[k];  // in-place calls (q_i -> q_i) read the source first
        s->apply_if(in, tgt.c[k], alpha_base, false, rp);
    }
}

void Ifherk::lin_sys(double alpha_k)
{
    divergence(r_i, cell_aux);
    s->apply_lgf(cell_aux.c[0], d_i.c[0], AMR2AMR, true, false);
    if (ib)
    {
        // lin_sys_with_ib_solve (ifherk.hpp:1451-1517)
        VField& fa2 = ib->face_aux2;
        copy(r_i, fa2, 1.0);
        gradient(d_i, face_aux);
        add(face_aux, fa2, -1.0);
        if (std::fabs(alpha_k) > 1e-14)
            for (int k = 0; k < 3; ++k)
            {
                int rp[3];
                mesh_relpos(MESH_FACE, k, rp);
                const Field in = fa2.c[k];
                s->apply_if(in, fa2.c[k], alpha_k, false, rp, IB2xIB);
            }
        std::vector<std::array<double, 3>> force = force_prev[stage_idx];
        const VField uin = fa2;
        ib->solve(uin, alpha_k, force, cg_threshold, cg_max_iter);
        if (write_prev_force) force_prev[stage_idx] = force;
        ib->pressure_correction(force, d_i);
        gradient(d_i, face_aux);
        ib->smearing(force, face_aux, false);
        add(face_aux, r_i, -1.0);
        if (std::fabs(alpha_k) > 1e-14) apply_if(r_i, u_i, alpha_k);
        else copy(r_i, u_i, 1.0);
        return;
    }
    gradient(d_i, face_aux);
    add(face_aux, r_i, -1.0);
    if (std::fabs(alpha_k) > 1e-14) apply_if(r_i, u_i, alpha_k);
    else copy(r_i, u_i, 1.0);
}

// pad_velocity<u, u>(true) (ifherk.hpp:1522-1573): the velocity is rebuilt
// from its vorticity through the stream function on the base level
void Ifherk::pad_velocity()
{
    const int bl = d->base_level;
    clean(u, true);
    up(u);
    clean(edge_aux, false);
    clean(stream_f, false);
    for (int l = bl; l < d->depth; ++l)
    {
        exchange(u, l);
        apply_op(*d, 3, {&u.c[0], &u.c[1], &u.c[2]}, {&edge_aux.c[0], &edge_aux.c[1], &edge_aux.c[2]}, l, 1.0,
                 true);
    }
    clean_leaf_correction_boundary(edge_aux, bl, true);
    for (int k = 0; k < 3; ++k) s->apply_lgf(edge_aux.c[k], stream_f.c[k], STREAM, true, false);
    // refresh_correction_only: curl_transpose on the base level only
    op_level(4, {&stream_f.c[0], &stream_f.c[1], &stream_f.c[2]}, {&u.c[0], &u.c[1], &u.c[2]}, bl, -1.0);
    down_to_correction(u);
}

// adapt_corr_time_step (ifherk.hpp:1206-1303): three projection stages with
// alpha = 0 and no nonlinear term; the IB solves start from the stage's
// previous force without replacing it (write_prev_force = false)
void Ifherk::adapt_corr_time_step()
{
    up_and_down(u);
    copy(u, q_i, 1.0);
    write_prev_force = false;
    // stage 1
    clean(g_i, false);
    clean(d_i, false);
    clean(cell_aux, false);
    clean(face_aux, false);
    copy(q_i, r_i, 1.0);
    stage_idx = 1;
    lin_sys(0.0);
    // stage 2
    clean(r_i, false);
    clean(d_i, false);
    clean(cell_aux, false);
    add(q_i, r_i, 1.0);
    up_and_down(u_i);
    stage_idx = 2;
    lin_sys(0.0);
    // stage 3
    clean(d_i, false);
    clean(cell_aux, false);
    clean(w_2, false);
    copy(q_i, r_i, 1.0);
    apply_if(r_i, r_i, 0.0);
    up_and_down(u_i);
    stage_idx = 3;
    lin_sys(0.0);
    write_prev_force = true;
    copy(u_i, u, 1.0);
    copy(d_i, p, 0.0);
}

void Ifherk::time_step()
{
    const double dx = d->dx_base;
    // ifherk.hpp:1093-1111: the velocity refresh replaces up_and_down(u)
    if (force_refresh || (T - T_last_vel_refresh) / (Re * dx * dx) * 3.3 > 7)
    {
        force_refresh = false;
        T_last_vel_refresh = T;
        pad_velocity();
        adapt_corr_time_step();
    }
    else
        up_and_down(u);
    copy(u, q_i, 1.0);
    // stage 1
    clean(g_i, false);
    clean(d_i, false);
    clean(cell_aux, false);
    clean(face_aux, false);
    nonlinear(u, g_i, coeff_a(1, 1) * (-dt));
    copy(q_i, r_i, 1.0);
    add(g_i, r_i, 1.0);
    stage_idx = 1;
    lin_sys(alpha[0]);
    // stage 2
    clean(r_i, false);
    clean(d_i, false);
    clean(cell_aux, false);
    add(g_i, face_aux, -1.0);
    copy(face_aux, w_1, -1.0 / dt / coeff_a(1, 1));
    apply_if(q_i, q_i, alpha[0]);
    apply_if(w_1, w_1, alpha[0]);
    add(q_i, r_i, 1.0);
    add(w_1, r_i, dt * coeff_a(2, 1));
    up_and_down(u_i);
    nonlinear(u_i, g_i, coeff_a(2, 2) * (-dt));
    add(g_i, r_i, 1.0);
    stage_idx = 2;
    lin_sys(alpha[1]);
    // stage 3
    clean(d_i, false);
    clean(cell_aux, false);
    clean(w_2, false);
    add(g_i, face_aux, -1.0);
    copy(face_aux, w_2, -1.0 / dt / coeff_a(2, 2));
    copy(q_i, r_i, 1.0);
    add(w_1, r_i, dt * coeff_a(3, 1));
    add(w_2, r_i, dt * coeff_a(3, 2));
    apply_if(r_i, r_i, alpha[1]);
    up_and_down(u_i);
    nonlinear(u_i, g_i, coeff_a(3, 3) * (-dt));
    add(g_i, r_i, 1.0);
    stage_idx = 3;
    lin_sys(alpha[2]);
    copy(u_i, u, 1.0);
    copy(d_i, p, 1.0 / coeff_a(3, 3) / dt);
    T += dt;
    // the next loop iteration resets old_correction to the correction flags
    for (Octant* o : d->octs) o->old_correction = false;
}
}  // namespace orc
