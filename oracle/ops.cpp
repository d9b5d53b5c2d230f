// ORACLE (test infrastructure): staggered mimetic block operators and the
// same-level buffer exchange, restating
//   include/iblgf/operators/operators.hpp:1386-1513 (laplace, gradient,
//     divergence, curl), :2416-2453 (curl_transpose), :2455-2531 (nonlinear)
//   include/iblgf/domain/mpi/haloCommunicator.hpp:63-107 (buffer exchange).
// Operators write the interior nodes of each block of a level; buffers are
// only read. Vector fields are three component fields (face: normal
// components x,y,z; edge: x,y,z).
#include <cmath>

#include "orc.hpp"

namespace orc
{
void buffer_exchange(Domain& d, Field& f, int level)
{
    const int Nb = d.Nb, e = d.e;
    const size_t B = (size_t)Nb * Nb * Nb;
    for (auto& kv : d.level_maps[level])
    {
        Octant* o = kv.second;
        double* dst = &f[o->idx * B];
        for (int ni = 0; ni < 27; ++ni)
        {
            Octant* n = o->neighbor[ni];
            if (!n || !n->has_data || n == o) continue;
            const double* sp = &f[n->idx * B];
            for (int k = 0; k < Nb; ++k)
                for (int j = 0; j < Nb; ++j)
                    for (int i = 0; i < Nb; ++i)
                    {
                        const int li = o->bbase[0] - 1 + i - n->bbase[0];
                        const int lj = o->bbase[1] - 1 + j - n->bbase[1];
                        const int lk = o->bbase[2] - 1 + k - n->bbase[2];
                        if (li < 0 || lj < 0 || lk < 0 || li >= e || lj >= e || lk >= e) continue;
                        dst[i + (size_t)Nb * (j + (size_t)Nb * k)] =
                            sp[(li + 1) + (size_t)Nb * ((lj + 1) + (size_t)Nb * (lk + 1))];
                    }
        }
    }
}

namespace
{
template<class F>
void for_blocks(Domain& d, int level, F&& f)
{
    for (int l = 0; l < (int)d.level_maps.size(); ++l)
    {
        if (level >= 0 && l != level) continue;
        for (auto& kv : d.level_maps[l])
        {
            const double dx = d.dx_base / std::pow(2.0, l - d.base_level);
            f(kv.second, dx);
        }
    }
}
}  // namespace

// op: 0 laplace, 1 gradient, 2 divergence, 3 curl, 4 curl_transpose, 5 nonlinear
void apply_op(Domain& d, int op, const std::vector<const Field*>& in, const std::vector<Field*>& out,
              int level, double scale, bool skip_correction)
{
    const int Nb = d.Nb;
    const size_t B = (size_t)Nb * Nb * Nb;
    for_blocks(d, level, [&](Octant* o, double dx) {
        if (skip_correction && o->correction) return;
        const size_t base = o->idx * B;
        auto at = [&](int c, int i, int j, int k) {
            return (*in[c])[base + i + (size_t)Nb * (j + (size_t)Nb * k)];
        };
        auto put = [&](int c, int i, int j, int k, double v) {
            (*out[c])[base + i + (size_t)Nb * (j + (size_t)Nb * k)] = v;
        };
        for (int k = 1; k < Nb - 1; ++k)
            for (int j = 1; j < Nb - 1; ++j)
                for (int i = 1; i < Nb - 1; ++i)
                {
                    if (op == 0)
                    {
                        double v = -6.0 * at(0, i, j, k) + at(0, i, j, k - 1) + at(0, i, j, k + 1) +
                                   at(0, i, j - 1, k) + at(0, i, j + 1, k) + at(0, i - 1, j, k) + at(0, i + 1, j, k);
                        put(0, i, j, k, v * (1.0 / (dx * dx)));
                    }
                    else if (op == 1)
                    {
                        const double fac = 1.0 / dx, s = at(0, i, j, k);
                        put(0, i, j, k, fac * (s - at(0, i - 1, j, k)));
                        put(1, i, j, k, fac * (s - at(0, i, j - 1, k)));
                        put(2, i, j, k, fac * (s - at(0, i, j, k - 1)));
                    }
                    else if (op == 2)
                    {
                        double v = -at(0, i, j, k) - at(1, i, j, k) - at(2, i, j, k) + at(0, i + 1, j, k) +
                                   at(1, i, j + 1, k) + at(2, i, j, k + 1);
                        put(0, i, j, k, v * (1.0 / dx));
                    }
                    else if (op == 3)
                    {
                        const double fac = 1.0 / dx;
                        put(0, i, j, k, fac * (at(2, i, j, k) - at(2, i, j - 1, k) - at(1, i, j, k) + at(1, i, j, k - 1)));
                        put(1, i, j, k, fac * (at(0, i, j, k) - at(0, i, j, k - 1) - at(2, i, j, k) + at(2, i - 1, j, k)));
                        put(2, i, j, k, fac * (at(1, i, j, k) - at(1, i - 1, j, k) - at(0, i, j, k) + at(0, i, j - 1, k)));
                    }
                    else if (op == 4)
                    {
                        const double fac = 1.0 / dx * scale;
                        put(0, i, j, k, fac * (at(1, i, j, k) - at(1, i, j, k + 1) + at(2, i, j + 1, k) - at(2, i, j, k)));
                        put(1, i, j, k, fac * (at(2, i, j, k) - at(2, i + 1, j, k) + at(0, i, j, k + 1) - at(0, i, j, k)));
                        put(2, i, j, k, fac * (at(0, i, j, k) - at(0, i, j + 1, k) + at(1, i + 1, j, k) - at(1, i, j, k)));
                    }
                    else
                    {
                        // in: face 0..2, edge 3..5
                        auto f = [&](int c, int a, int b, int cc) { return at(c, i + a, j + b, k + cc); };
                        auto w = [&](int c, int a, int b, int cc) { return at(3 + c, i + a, j + b, k + cc); };
                        put(0, i, j, k,
                            0.25 * (w(1, 0, 0, 0) * (f(2, 0, 0, 0) + f(2, -1, 0, 0)) +
                                    w(1, 0, 0, 1) * (f(2, 0, 0, 1) + f(2, -1, 0, 1)) -
                                    w(2, 0, 0, 0) * (f(1, 0, 0, 0) + f(1, -1, 0, 0)) -
                                    w(2, 0, 1, 0) * (f(1, 0, 1, 0) + f(1, -1, 1, 0))));
                        put(1, i, j, k,
                            0.25 * (w(2, 0, 0, 0) * (f(0, 0, 0, 0) + f(0, 0, -1, 0)) +
                                    w(2, 1, 0, 0) * (f(0, 1, 0, 0) + f(0, 1, -1, 0)) -
                                    w(0, 0, 0, 0) * (f(2, 0, 0, 0) + f(2, 0, -1, 0)) -
                                    w(0, 0, 0, 1) * (f(2, 0, 0, 1) + f(2, 0, -1, 1))));
                        put(2, i, j, k,
                            0.25 * (w(0, 0, 0, 0) * (f(1, 0, 0, 0) + f(1, 0, 0, -1)) +
                                    w(0, 0, 1, 0) * (f(1, 0, 1, 0) + f(1, 0, 1, -1)) -
                                    w(1, 0, 0, 0) * (f(0, 0, 0, 0) + f(0, 0, 0, -1)) -
                                    w(1, 1, 0, 0) * (f(0, 1, 0, 0) + f(0, 1, 0, -1))));
                    }
                }
    });
}

}  // namespace orc
