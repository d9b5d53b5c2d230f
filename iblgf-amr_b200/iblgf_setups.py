"""Problem setups that call the LGF-FMM path: domain configurations, refinement
predicates and source / exact fields, in the roles the reference's setups and
tests play (tests/poisson/vortexrings.hpp, tests/conv_test/ffmTest.cpp).

Everything here is host-side numpy that produces inputs for the solver; the
solver itself lives in the CUDA library. Fields are numpy arrays of shape
(n_octants, Nb, Nb, Nb) indexed [octant][z][y][x] (x fastest in memory), i.e.
the reference's column-major Nb^3 blocks with their one-cell buffers.
"""
import numpy as np


# --------------------------------------------------------------------------
# Vortex-ring manufactured solution (tests/poisson/vortexrings.hpp:50-145)
def vortex_ring_psi_lap(x, y, z, R, c1, c2):
    """psi = c1 exp(-c2 / (1 - t^2)), t = dist(ring)/R, and its analytic
    Laplacian (chain rule in s = t^2), zero outside the torus t >= 1."""
    r = np.sqrt(x * x + y * y)
    s = ((r - R) ** 2 + z * z) / R ** 2
    inside = s < 1.0
    sc = np.where(inside, s, 0.0)
    om = 1.0 - sc
    psi = np.where(inside, c1 * np.exp(-c2 / om), 0.0)
    ps = psi * (-c2 / om ** 2)
    pss = psi * (c2 * c2 / om ** 4 - 2.0 * c2 / om ** 3)
    rr = np.where(r > 0, r, 1.0)
    lap = ps * (6.0 / R ** 2 - 2.0 / (rr * R)) + pss * 4.0 * sc / R ** 2
    return psi, np.where(inside, lap, 0.0)


class VortexRingPoisson:
    """tests/poisson/configs/config_1_lv_{0,1}: 192^3 bounding box, 96^3 block
    region of 6^3 blocks, Lx = 2.5, one ring R = 0.125, c1 = 1e6, c2 = 15,
    refinement_factor 0.125, EXP_LInf 0.0116450 (nLevels 0) / 1e-2 (nLevels 1).
    """

    def __init__(self, n_levels=0, block_extent=6):
        self.bd_base = (-96, -96, -96)
        self.bd_extent = (192, 192, 192)
        self.block_extent = block_extent
        self.dx_base = 2.5 / 192.0
        self.blocks = [((-48, -48, -48), (96, 96, 96))]
        self.n_levels = n_levels
        self.R, self.c1, self.c2 = 0.125, 1.0e6, 15.0
        self.refinement_factor = 0.125
        self.exp_linf = 0.0116450 if n_levels == 0 else 1e-2
        # bounding box centre in base cells, (max - min) / 2 + min
        self.center = (self.bd_base[0] + self.bd_extent[0] - 1 - self.bd_base[0]) / 2.0 + self.bd_base[0]
        _, lap = vortex_ring_psi_lap(np.array([self.R]), np.array([0.0]), np.array([0.0]),
                                     self.R, self.c1, self.c2)
        self.source_max = abs(float(lap[0]))

    def _xyz(self, base, n, rl, lo=0):
        sc = 2 ** rl
        dxl = self.dx_base / sc
        i = np.arange(n) + lo
        c = self.center * sc
        return ((base[0] + i - c + 0.5) * dxl, (base[1] + i - c + 0.5) * dxl,
                (base[2] + i - c + 0.5) * dxl)

    def predicate(self, base, extent, rl, diff_level):
        """vortexrings.hpp:481-517: refine if |source| exceeds
        source_max * refinement_factor^diff_level on the block grown by 2."""
        e = extent[0]
        X, Y, Z = self._xyz(base, e + 4, rl, lo=-2)
        _, lap = vortex_ring_psi_lap(X[:, None, None], Y[None, :, None], Z[None, None, :],
                                     self.R, self.c1, self.c2)
        return bool((np.abs(lap) > self.source_max * self.refinement_factor ** diff_level).any())

    def fields(self, octs):
        """Source on every leaf and the exact solution, interior nodes only."""
        Nb, e = self.block_extent + 2, self.block_extent
        src = np.zeros((octs.n, Nb, Nb, Nb))
        ex = np.zeros_like(src)
        for o in range(octs.n):
            if not octs.leaf[o]:
                continue
            rl = int(octs.levels[o]) - octs.base_level
            X, Y, Z = self._xyz(octs.bbase[o], e, rl)
            p, lap = vortex_ring_psi_lap(X[None, None, :], Y[None, :, None], Z[:, None, None],
                                         self.R, self.c1, self.c2)
            src[o, 1:-1, 1:-1, 1:-1] = lap
            ex[o, 1:-1, 1:-1, 1:-1] = p
        return src, ex

    def finest_linf(self, octs, num, ex):
        L = octs.depth - 1
        err = 0.0
        for o in range(octs.n):
            if octs.levels[o] != L or not octs.leaf[o] or octs.correction[o]:
                continue
            err = max(err, float(np.abs(num[o, 1:-1, 1:-1, 1:-1] - ex[o, 1:-1, 1:-1, 1:-1]).max()))
        return err


# --------------------------------------------------------------------------
# Gaussian-source Poisson problems (the LGF-FMM benchmark workloads)
class GaussianPoisson:
    """Unbounded 3-D Poisson problem with a sum-of-Gaussians source sampled at
    cell centres, x = (i + 0.5) dx_level in level cell units, origin at the
    centre of the block region.

    uniform_64:  4x4x4 blocks of 16^3 cells (64^3 cells), dx = 1, one level;
                 source = +exp(-|x-c+|^2/32) - exp(-|x-c-|^2/32), c = (+-12,0,0).
    amr_3level:  8x8x8 base blocks of 16^3 cells, two refinement levels where
                 |f| > 1e-3 max|f| (base -> 1) and > 1e-2 max|f| (1 -> 2) on
                 the block grown by 2 cells; source = the uniform_64 pair plus
                 16 Gaussians, sigma ~ U[2, 6] cells, amplitude ~ U[-1, 1],
                 centres uniform in the inner 50% of the block region
                 (numpy PCG64, seed 20261203).
    """

    def __init__(self, name="uniform_64", block_extent=16, seed=20261203):
        self.name = name
        self.block_extent = block_extent
        self.dx_base = 1.0
        g = [(1.0, 4.0, (12.0, 0.0, 0.0)), (-1.0, 4.0, (-12.0, 0.0, 0.0))]
        n_random, sig_range = 0, (2.0, 6.0)
        if name == "uniform_64":
            half = 32
            self.n_levels = 0
        elif name in ("amr_3level", "amr_2level"):
            # amr_2level: the same source and base mesh with one refinement
            # level (a medium-size case for profiling)
            half = 64
            self.n_levels = 2 if name == "amr_3level" else 1
            n_random = 16
        elif name in ("uniform_small", "amr_small"):
            # reduced parity cases: 4x4x4 base blocks of 6^3 cells
            self.block_extent = block_extent = 6
            half = 12
            g = [(1.0, 1.5, (4.5, 0.0, 0.0)), (-1.0, 1.5, (-4.5, 0.0, 0.0))]
            self.n_levels = 0 if name == "uniform_small" else 2
            n_random, sig_range = (6 if name == "amr_small" else 0), (0.8, 2.0)
        else:
            raise ValueError(name)
        if n_random:
            rng = np.random.Generator(np.random.PCG64(seed))
            for _ in range(n_random):
                sig = rng.uniform(*sig_range)
                amp = rng.uniform(-1.0, 1.0)
                c = rng.uniform(-half / 2.0, half / 2.0, size=3)
                g.append((amp, sig, tuple(c)))
        self.gaussians = g
        self.bd_base = (-2 * half,) * 3
        self.bd_extent = (4 * half,) * 3
        self.blocks = [((-half,) * 3, (2 * half,) * 3)]
        self.fmax = self._fmax()

    def f(self, X, Y, Z):
        out = np.zeros(np.broadcast(X, Y, Z).shape)
        for a, s, c in self.gaussians:
            out += a * np.exp(-((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2) / (2.0 * s * s))
        return out

    def _fmax(self):
        x = np.arange(-self.blocks[0][1][0] // 2, self.blocks[0][1][0] // 2) + 0.5
        return float(np.abs(self.f(x[:, None, None], x[None, :, None], x[None, None, :])).max())

    def _xyz(self, base, n, rl, lo=0):
        dxl = self.dx_base / 2 ** rl
        i = np.arange(n) + lo
        return ((base[0] + i + 0.5) * dxl, (base[1] + i + 0.5) * dxl, (base[2] + i + 0.5) * dxl)

    def predicate(self, base, extent, rl, diff_level):
        e = extent[0]
        X, Y, Z = self._xyz(base, e + 4, rl, lo=-2)
        thresh = self.fmax * (1e-3 if rl == 0 else 1e-2)
        return bool((np.abs(self.f(X[:, None, None], Y[None, :, None], Z[None, None, :])) > thresh).any())

    def fields(self, octs):
        Nb, e = self.block_extent + 2, self.block_extent
        src = np.zeros((octs.n, Nb, Nb, Nb))
        for o in range(octs.n):
            if not octs.leaf[o]:
                continue
            rl = int(octs.levels[o]) - octs.base_level
            X, Y, Z = self._xyz(octs.bbase[o], e, rl)
            src[o, 1:-1, 1:-1, 1:-1] = self.f(X[None, None, :], Y[None, :, None], Z[:, None, None])
        return src

    def n_cells(self, octs):
        """Cells per solve: leaf blocks (correction leaves included) x e^3,
        the reference's get_nPoints (domain.hpp:1218-1248)."""
        return int(np.count_nonzero(octs.leaf)) * self.block_extent ** 3


class ImpulseFmm:
    """tests/conv_test/configs/configFFMTest: 48^3 domain, block_extent 6,
    nLevels 0; unit impulse at local (1,1,1) of the first non-correction leaf
    in key order; the base-level FMM must reproduce LGF_GL::get."""

    def __init__(self, dx_base=1.0):
        self.bd_base = (-24, -24, -24)
        self.bd_extent = (48, 48, 48)
        self.block_extent = 6
        self.dx_base = dx_base
        self.blocks = [((-24, -24, -24), (48, 48, 48))]
        self.n_levels = 0

    def source(self, octs):
        Nb = self.block_extent + 2
        src = np.zeros((octs.n, Nb, Nb, Nb))
        order = np.argsort(octs.keys, kind="stable")
        i0 = next(int(i) for i in order if octs.leaf[i] and not octs.correction[i])
        src[i0, 1, 1, 1] = 1.0
        return src, i0, np.array(octs.bbase[i0])


class VortexRingNS:
    """Vortex-ring flow for the IF-HERK time step (the incompressible NS
    setups, e.g. setups/ns_amr_lgf: one ring of radius R = 1 in the z = 0
    plane, Gaussian core sigma = 0.2 R, Re = 1000).

    The initial face velocity is the curl of the vector potential
    A = a0 exp(-d^2 / sigma_A^2) (-y, x, 0), d = distance to the core circle,
    evaluated at the face centres (synthetic stand-in for the reference's
    vorticity-to-velocity initialisation; peak speed about Gamma / (2 pi sigma)
    * 0.64 for circulation Gamma = 1). The mesh refines where the core factor
    exp(-d^2 / sigma^2) on the block grown by 2 cells exceeds thresh[rl].

    c4:    dx_base = R/8, 16^3 blocks, box +-3R, two refinement levels
           (dx_finest = R/32), 3 mesh levels
    small: dx_base = R/4, 6^3 blocks, box +-3R, one refinement level (parity)
    """

    def __init__(self, name="c4"):
        self.name = name
        self.R, self.sigma, self.Re, self.cfl = 1.0, 0.2, 1000.0, 0.35
        if name == "c4":
            self.block_extent, self.dx_base, self.n_levels = 16, 1.0 / 8, 2
            self.thresh = (2e-3, 2e-2)
        elif name == "small":
            self.block_extent, self.dx_base, self.n_levels = 6, 1.0 / 4, 1
            self.thresh = (1e-2,)
        else:
            raise ValueError(name)
        half = int(round(3.0 * self.R / self.dx_base))
        half = -(-half // self.block_extent) * self.block_extent
        self.bd_base = (-2 * half,) * 3
        self.bd_extent = (4 * half,) * 3
        self.blocks = [((-half,) * 3, (2 * half,) * 3)]
        self.sigma_a = 1.5 * self.sigma
        self.a0 = 1.0
        self.a0 = 0.5 / self._umax_probe()

    def _core(self, X, Y, Z):
        rho = np.sqrt(X * X + Y * Y)
        return np.exp(-((rho - self.R) ** 2 + Z * Z) / self.sigma ** 2)

    def _A(self, X, Y, Z):
        rho = np.sqrt(X * X + Y * Y)
        g = self.a0 * np.exp(-((rho - self.R) ** 2 + Z * Z) / self.sigma_a ** 2)
        return -Y * g, X * g, np.zeros_like(g)

    def velocity(self, X, Y, Z, comp, h=1e-6):
        """Component comp of curl A by central differences of the analytic A."""
        def d(axis, k):
            e = [0.0, 0.0, 0.0]
            e[axis] = h
            p = self._A(X + e[0], Y + e[1], Z + e[2])[k]
            m = self._A(X - e[0], Y - e[1], Z - e[2])[k]
            return (p - m) / (2 * h)
        if comp == 0:
            return d(1, 2) - d(2, 1)
        if comp == 1:
            return d(2, 0) - d(0, 2)
        return d(0, 1) - d(1, 0)

    def _umax_probe(self):
        x = np.linspace(-2.0, 2.0, 81)
        X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
        return float(max(np.abs(self.velocity(X, Y, Z, k)).max() for k in range(3)))

    def predicate(self, base, extent, rl, diff_level):
        e = extent[0]
        dxl = self.dx_base / 2 ** rl
        i = np.arange(e + 4) - 2
        x, y, z = ((base[a] + i + 0.5) * dxl for a in range(3))
        g = self._core(x[:, None, None], y[None, :, None], z[None, None, :])
        return bool(rl < len(self.thresh) and (g > self.thresh[rl]).any())

    def initial_velocity(self, octs):
        """(3, n, Nb, Nb, Nb) face velocity on every block, buffers included:
        component d sits on the cell face normal to d at the lower side,
        x_d = (b_d + i - 1) dx, the other coordinates at cell centres."""
        Nb = self.block_extent + 2
        u = np.zeros((3, octs.n, Nb, Nb, Nb))
        i = np.arange(Nb) - 1.0
        for o in range(octs.n):
            rl = int(octs.levels[o]) - octs.base_level
            dxl = self.dx_base / 2 ** rl
            b = octs.bbase[o]
            for comp in range(3):
                c = [(b[a] + i + (0.0 if a == comp else 0.5)) * dxl for a in range(3)]
                u[comp, o] = self.velocity(c[0][None, None, :], c[1][None, :, None], c[2][:, None, None], comp)
        return u

    def dt(self):
        dx_finest = self.dx_base / 2 ** self.n_levels
        return self.cfl * dx_finest / 0.5


class BatchPoisson:
    """Batch of independent unbounded Poisson problems of uneven size.

    c3:    256 problems, 16^3-cell blocks, dx = 1; block count per problem
           n = floor(exp(U[0, ln 64])) clipped to [1, 64] (log-uniform); the
           n blocks fill the most compact near-cube box a x b x c (x fastest),
           a = ceil(n^(1/3)), b = ceil(sqrt(n / a)), c = ceil(n / (a b));
           source = 4 Gaussians per problem, sigma ~ U[2, 6] cells, amplitude
           ~ U[-1, 1], centres uniform in the problem's block box
           (numpy PCG64, seed 20261203); one mesh level.
    small: 6 problems of 1..27 blocks of 6^3 cells (parity case).
    """

    def __init__(self, name="c3", seed=20261203):
        self.name = name
        rng = np.random.Generator(np.random.PCG64(seed))
        if name == "c3":
            self.block_extent, n_prob, nmax, sig = 16, 256, 64, (2.0, 6.0)
            counts = [int(min(max(np.floor(np.exp(rng.uniform(0.0, np.log(nmax)))), 1), nmax))
                      for _ in range(n_prob)]
        elif name == "small":
            self.block_extent, sig = 6, (0.8, 2.0)
            counts = [1, 27, 5, 12, 2, 8]
        else:
            raise ValueError(name)
        self.dx_base = 1.0
        e = self.block_extent
        self.problems = []
        for n in counts:
            a = int(np.ceil(round(n ** (1.0 / 3.0), 9)))
            b = int(np.ceil(np.sqrt(n / a)))
            c = int(np.ceil(n / (a * b)))
            dims = (a, b, c)
            start = [-((d + 1) // 2) * e for d in dims]
            blocks = []
            for i in range(n):
                pos = (i % a, (i // a) % b, i // (a * b))
                blocks.append((tuple(start[k] + pos[k] * e for k in range(3)), (e, e, e)))
            m = 1
            while m < max(dims):
                m *= 2
            half = max(m * e // 2, e)
            lo = np.array(start, float)
            hi = lo + np.array(dims, float) * e
            g = []
            for _ in range(4):
                s = rng.uniform(*sig)
                amp = rng.uniform(-1.0, 1.0)
                ctr = tuple(rng.uniform(lo[k], hi[k]) for k in range(3))
                g.append((amp, s, ctr))
            self.problems.append({"bd_base": (-2 * half,) * 3, "bd_extent": (4 * half,) * 3, "blocks": blocks,
                                  "gaussians": g, "n_blocks": n})

    @staticmethod
    def _f(gauss, X, Y, Z):
        out = np.zeros(np.broadcast(X, Y, Z).shape)
        for a, s, c in gauss:
            out += a * np.exp(-((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2) / (2.0 * s * s))
        return out

    def fields(self, octs, i):
        """Source of problem i on its leaves (interior nodes), octs = that
        problem's octants (a BatchSolver problem view or an oracle Domain)."""
        e = self.block_extent
        Nb = e + 2
        src = np.zeros((octs.n, Nb, Nb, Nb))
        x = np.arange(e) + 0.5
        for o in range(octs.n):
            if not octs.leaf[o]:
                continue
            b = octs.bbase[o]
            src[o, 1:-1, 1:-1, 1:-1] = self._f(self.problems[i]["gaussians"], (b[0] + x)[None, None, :],
                                               (b[1] + x)[None, :, None], (b[2] + x)[:, None, None])
        return src

    def n_cells(self, octs):
        return int(np.count_nonzero(octs.leaf)) * self.block_extent ** 3


class SphereIB:
    """Immersed-boundary sphere (the reference's geometry=sphere, ib.hpp:179-210:
    R = 0.5 at the origin, Fibonacci points at spacing ibph * dx_ib) in a
    block-refined box; the IB lives on the finest level.

    small: 6^3 blocks, dx_base = 1/8, box +-1.5, one refinement level around
           the sphere (dx_ib = 1/16), ibph 1.5 (413 points), Re = 300
    c5:    16^3 blocks, dx_base = 1/10, box +-3.2 x +-3.2 x [-3.2, 6.4) with a
           wake, two refinement levels (dx_ib = D/40), ibph 1.7 (2009 points),
           Re = 300
    """

    def __init__(self, name="small"):
        self.name, self.Re = name, 300.0
        if name == "small":
            self.block_extent, self.dx_base, self.n_levels, self.ibph = 6, 1.0 / 8, 1, 1.5
            lo, hi = (-12, -12, -12), (12, 12, 12)
            self.radii = (1.1,)
        elif name == "c5":
            self.block_extent, self.dx_base, self.n_levels, self.ibph = 16, 1.0 / 10, 2, 1.7
            lo, hi = (-32, -32, -32), (64, 32, 32)
            self.radii = (1.6, 1.0)
        else:
            raise ValueError(name)
        e = self.block_extent
        self.blocks = [(lo, tuple(h - l for l, h in zip(lo, hi)))]
        m = 1
        while m * e < max(max(abs(v) for v in lo), max(abs(v) for v in hi)):
            m *= 2
        half = m * e
        self.bd_base = (-2 * half,) * 3
        self.bd_extent = (4 * half,) * 3

    def points(self):
        import oracle_lib as O  # noqa: F401  (tests only)
        raise NotImplementedError

    def predicate(self, base, extent, rl, diff_level):
        """Refine blocks (grown by 2 cells) that reach within radii[rl] of the
        sphere centre; the c5 wake extends the base-level region downstream."""
        if rl >= len(self.radii):
            return False
        dxl = self.dx_base / 2 ** rl
        lo = [(base[d] - 2) * dxl for d in range(3)]
        hi = [(base[d] + extent[d] + 2) * dxl for d in range(3)]
        r = self.radii[rl]
        if self.name == "c5" and rl == 0:
            # wake: a cylinder of radius r behind the sphere up to x = 4
            q = [min(max(0.0, lo[1]), hi[1]), min(max(0.0, lo[2]), hi[2])]
            if hi[0] > -r and lo[0] < 4.0 and q[0] ** 2 + q[1] ** 2 < r * r:
                return True
        c = [min(max(0.0, lo[d]), hi[d]) for d in range(3)]
        return c[0] ** 2 + c[1] ** 2 + c[2] ** 2 < r * r

    def velocity(self, octs, U=(1.0, 0.0, 0.0), seed=5):
        """Face velocity: the uniform stream U plus a smooth seeded
        perturbation, on every block (buffers included)."""
        rng = np.random.Generator(np.random.PCG64(seed))
        k = rng.uniform(0.5, 2.0, size=(3, 3))
        Nb = self.block_extent + 2
        u = np.zeros((3, octs.n, Nb, Nb, Nb))
        i = np.arange(Nb) - 1.0
        for o in range(octs.n):
            rl = int(octs.levels[o]) - octs.base_level
            dxl = self.dx_base / 2 ** rl
            b = octs.bbase[o]
            for c in range(3):
                x = [(b[a] + i + (0.0 if a == c else 0.5)) * dxl for a in range(3)]
                X, Y, Z = x[0][None, None, :], x[1][None, :, None], x[2][:, None, None]
                u[c, o] = U[c] + 0.1 * np.sin(k[c, 0] * X) * np.cos(k[c, 1] * Y) * np.cos(k[c, 2] * Z)
        return u


# ----------------------------------------------------------------- adaptation
def key_parent(k):
    """Parent Morton key (octree/key.hpp parent(): coordinate bits of level
    l - 1, level field l - 1)."""
    k = int(k)
    lv = (k >> 2) & 31
    if lv == 0:
        return k
    m = 0 if lv - 1 <= 0 else ((1 << (3 * (lv - 1))) - 1) << (64 - 3 * (lv - 1))
    return ((m & k) | ((lv - 1) << 2)) + 1


def update_source_max(source_max, block_rms, all_time_max=False):
    """Ifherk::update_source_max (ifherk.hpp:401-426): the largest block RMS
    of the field, blended with (or maxed against) the previous value, at least
    1e-2."""
    new = float(np.max(block_rms)) if len(block_rms) else 0.0
    out = max(source_max, new) if all_time_max else 0.5 * (source_max + new)
    return max(out, 1e-2)


def adapt_level_change(keys, levels, flags, base_level, cell_aux_max, correction_max, edge_aux_max, source_max,
                       n_level_refinement, refinement_factor=0.125, base_threshold=1e-4, hard_max_level=None,
                       ib_flags=None, n_ib_add_level=0):
    """The adapt condition of the reference's NS setup
    (tests/ns_amr_lgf/ns_amr_lgf.hpp:402-489): per-octant block max-norms
    (iblgf_block_norms) of cell_aux, correction_tmp and edge_aux against
    source_max = (cell, vorticity); returns the attempts (keys, level change)
    for iblgf_adapt. Leaves ask for refinement when the field is within the
    refinement_factor^k band of source_max for a deeper level, for deletion
    when it falls below the band by the deletion factor 0.7; correction blocks
    (non-leaf) ask through their parent's key."""
    hard = n_level_refinement if hard_max_level is None else hard_max_level
    ib = np.zeros(len(keys), np.int32) if ib_flags is None else np.asarray(ib_flags)
    out_k, out_l = [], []

    def field_change(o, field_max, smax, base_thr):
        rl = int(levels[o]) - base_level
        if (ib[o] & 1) and (flags[o] & 1):
            return 1 if rl < n_level_refinement + n_ib_add_level else 0
        smax *= 1.05
        if field_max < 1e-10:
            return -1
        deletion_factor = 0.7
        lr = np.log(field_max / smax)
        l_aim = int(np.ceil(n_level_refinement - lr / np.log(refinement_factor)))
        l_del = int(np.ceil(n_level_refinement - ((lr - np.log(deletion_factor)) / np.log(refinement_factor))))
        l_aim = min(l_aim, hard)
        if rl == 0 and base_thr:
            if field_max > smax * base_threshold:
                l_aim = max(l_aim, 0)
            if field_max > smax * base_threshold * deletion_factor:
                l_del = max(l_del, 0)
        if ib[o] & 1:
            return 0
        if l_aim - rl > 0:
            return 1
        if l_del - rl < 0:
            return -1
        return 0

    for o in range(len(keys)):
        leaf, corr = bool(flags[o] & 1), bool(flags[o] & 2)
        if not leaf and not corr:
            continue
        if leaf and corr:
            continue
        l1 = l2 = l3 = -1
        if leaf and not corr:
            l1 = field_change(o, cell_aux_max[o], source_max[0], True)
            l3 = field_change(o, edge_aux_max[o], source_max[1], False)
        if corr and not leaf:
            l2 = field_change(o, correction_max[o], source_max[0], False)
        lv = max(l1, l2, l3)
        if lv != 0:
            if leaf and not corr:
                out_k.append(int(keys[o]))
                out_l.append(lv)
            elif corr and not leaf and l2 > 0:
                out_k.append(key_parent(keys[o]))
                out_l.append(l2)
    return np.array(out_k, np.uint64), np.array(out_l, np.int32)


class NsAmrLgfTest:
    """The reference's NS test (tests/ns_amr_lgf/configs): one fat vortex ring
    R = 0.5 in the z = 0 plane (vortex_ring_vor_fat_ic, ns_amr_lgf.hpp:588-612),
    Re = 1000, domain (-24..23)^3 base cells in blocks of 6^3, cfl 0.35, to
    T = 0.35:
      config 0: dx_base 0.25, no refinement, dt = dx_base cfl = 0.0875, 4 steps
      config 1: dx_base 0.5, one refinement level where the vorticity on the
                block grown by 2 cells exceeds w_max (1/8)^diff_level
                (refinement, :759-818), dt = 0.0875 on the fine level, 4 steps
    The velocity starts from the vorticity through the stream function
    (initialize, :491-575): vorticity on the edges, a Poisson solve per
    component, curl_transpose with scale -1. The test's pass marks (EXP_LInf)
    are 1e-2 and 3e-4 on the finest level's largest |u_x - u_ref,x|."""

    def __init__(self, config=1):
        self.config = config
        self.bd_base, self.bd_extent = (-24,) * 3, (48,) * 3
        self.block_extent = 6
        self.blocks = [((-24,) * 3, (48,) * 3)]
        self.R, self.Re, self.cfl = 0.5, 1000.0, 0.35
        self.refinement_factor = 0.125
        if config == 0:
            self.dx_base, self.n_levels, self.base_steps, self.exp_linf = 0.25, 0, 4, 1e-2
        else:
            self.dx_base, self.n_levels, self.base_steps, self.exp_linf = 0.5, 1, 2, 3e-4
        dt_base = self.dx_base * self.cfl
        self.dt = dt_base / 2 ** self.n_levels
        self.steps = self.base_steps * 2 ** self.n_levels
        self.T_end = self.base_steps * dt_base

    def predicate(self, base, extent, rl, diff_level):
        e = extent[0]
        dxl = self.dx_base / 2 ** rl
        w_max = abs(float(self.vorticity(np.array(self.R), np.array(0.0), np.array(0.0), 1)))
        thr = w_max * self.refinement_factor ** diff_level
        i = np.arange(-2, e + 2)
        c = [base[a] + i for a in range(3)]
        for comp in range(3):
            pos = [(c[a] + (0.5 if a == comp else 0.0)) * dxl for a in range(3)]
            w = self.vorticity(pos[0][:, None, None], pos[1][None, :, None], pos[2][None, None, :], comp)
            if (np.abs(w) > thr).any():
                return True
        return False

    def vorticity(self, x, y, z, comp):
        alpha = 0.54857674
        R2 = self.R * self.R
        r = np.sqrt(x * x + y * y)
        s2 = z * z + (r - self.R) ** 2
        theta = np.arctan2(y, x)
        with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
            w = alpha / R2 * np.exp(-4.0 * s2 / (R2 - s2))
        w = np.where(s2 >= R2, 0.0, w)
        if comp == 0:
            return -w * np.sin(theta)
        if comp == 1:
            return w * np.cos(theta)
        return np.zeros_like(w)

    def initial_vorticity(self, octs):
        """(3, n, Nb, Nb, Nb) edge vorticity on every node: edge component d at
        ((i + 1/2 [d = x]) dx, (j + 1/2 [d = y]) dx, (k + 1/2 [d = z]) dx), i, j,
        k global cell indices of the octant's level (the domain centre is the
        origin, ns_amr_lgf.hpp:500-540)."""
        Nb = self.block_extent + 2
        w = np.zeros((3, octs.n, Nb, Nb, Nb))
        i = np.arange(Nb) - 1.0
        for o in range(octs.n):
            rl = int(octs.levels[o]) - octs.base_level
            dxl = self.dx_base / 2 ** max(rl, 0)
            b = octs.bbase[o]
            for comp in range(3):
                c = [(b[a] + i + (0.5 if a == comp else 0.0)) * dxl for a in range(3)]
                w[comp, o] = self.vorticity(c[0][None, None, :], c[1][None, :, None], c[2][:, None, None], comp)
        return w
