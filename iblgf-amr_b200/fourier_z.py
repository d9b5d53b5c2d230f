"""Fourier-in-z solves on a uniform 2-D cell grid through the 2-D Helmholtz
lattice Green's function (Solver.helm2d_apply, lgf::Helmholtz<2>).

The reference's z-periodic setups (PoissonSolver::apply_lgf_and_helm,
include/iblgf/solver/poisson/poisson.hpp:173-219) transform the fields along
z, solve one 2-D problem per z mode with the Helmholtz kernel of that mode's
wave number (c = k 2 pi dx / L_z, poisson.hpp:107-112) and the 2-D Laplace
kernel for mode 0, and transform back. Here the 2-D problems are solved
exactly on a uniform grid (every source cell with every target cell, on the
device; mode 0 with the 2-D Laplace LGF, c = 0); the reference's 2-D quadtree
FMM, which approximates the same sums on an adaptive mesh, is not part of
this library. Mode 0's solution is the unbounded one (it grows like the log
of the distance when the source's total is not zero).
"""
import numpy as np


def mode_wave_numbers(nz, z_operator="second_order"):
    """c_k per z mode k = 0 .. nz-1 for unit spacing: 'second_order' for the
    three-point z Laplacian (c_k^2 = 2 - 2 cos(2 pi k / nz)), 'spectral' for
    the exact z derivative (c_k = 2 pi min(k, nz - k) / nz)."""
    k = np.arange(nz)
    if z_operator == "second_order":
        return 2.0 * np.abs(np.sin(np.pi * k / nz))
    if z_operator == "spectral":
        return 2.0 * np.pi * np.minimum(k, nz - k) / nz
    raise ValueError("z_operator must be 'second_order' or 'spectral'")


def solve(solver, f, z_operator="second_order"):
    """u with (Delta_xy + D_zz) u = f on the unbounded x-y plane, periodic
    in z, unit spacing; f has shape (nz, ny, nx)."""
    f = np.asarray(f, dtype=np.float64)
    nz = f.shape[0]
    fh = np.fft.fft(f, axis=0)
    ck = mode_wave_numbers(nz, z_operator)
    uh = np.zeros_like(fh)
    for k in range(nz):
        uh[k] = solver.helm2d_apply(ck[k], fh[k].real) + 1j * solver.helm2d_apply(ck[k], fh[k].imag)
    return np.fft.ifft(uh, axis=0).real


def refined_modes(n_modes, ref_level_up):
    """The modes the _refined operator forms compute (operators.hpp:1653-1722,
    1839-1887, 2125-2176): the first n_modes / 2^r; like the reference, an
    n_modes that 2^r does not divide is an error."""
    d = 1 << int(ref_level_up)
    if n_modes % d:
        raise ValueError("number of modes not divisible by 2^ref_level_up")
    return range(n_modes // d)


def one_mode_planes(mode, planes_per_mode=3):
    """The z planes nonlinear_helmholtz_oneMode computes (operators.hpp:2776-2831)."""
    return range(mode * planes_per_mode, (mode + 1) * planes_per_mode)


def refined_planes(n_planes, ref_level_up):
    """The z planes nonlinear_helmholtz_refined computes (operators.hpp:2840-2895):
    every 2^r-th."""
    return range(0, n_planes, 1 << int(ref_level_up))
