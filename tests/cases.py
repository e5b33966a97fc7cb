"""Small problem definitions shared by the parity tests.

Each builder returns a ``prob`` dict for ``starmap_init``.  Sizes are chosen so
that the numpy oracle finishes in well under a second; together the cases
cover 1D/2D/3D, both boundary conditions (also mixed per axis), odd and
unequal grid sizes, scalar and field coefficients, isotropic and anisotropic
scattering, sources on one or all moments, the three filter positions, P_N
and SP_N closures, time-dependent sources and materials, and output times.
"""
import numpy as np

from starmap_b200 import configs


def smooth(a, b, c):
    return lambda x, y: a + b * np.sin(2.1 * x + 0.3) * np.cos(1.7 * y - 0.2) + c * x * y


def lin_p7_periodic():
    return configs.linesource(n=20, n_mom=7, tfinal=2.5)


def lattice_p5_substep():
    return configs.lattice(n=21, n_mom=5, tfinal=5.0, f_position="substep")


def lattice_p4_full():
    return configs.lattice(n=14, n_mom=4, tfinal=6.0, f_position="full")


def lattice_p6_nofilter():
    return configs.lattice(n=14, n_mom=6, tfinal=5.0, f_position="")


def odd_mixed_bc():
    return dict(name="odd", closure="P", n_mom=3, ax=[-1.0, 1.2, -0.7, 0.9], n=[7, 5], bc=[0, 1],
                ic=lambda x, y, k: np.exp(-3 * (x ** 2 + (y - 0.1) ** 2)) * (1.0 / k) + 0.01 * k * x,
                sigma_a=smooth(0.3, 0.2, 0.1), sigma_s0=smooth(1.0, 0.3, -0.05),
                source=lambda x, y, t, k: np.exp(-4 * (x ** 2 + y ** 2)) * (0.5 if k == 1 else 0.05 / k),
                tfinal=3.0, t_plot=[0.0, 3.0], cn=0.9, quiet=True)


def aniso_2d():
    return dict(name="aniso", closure="P", n_mom=4, ax=[0, 1, 0, 1], n=[9, 8], bc=[1, 0],
                ic=lambda x, y: np.exp(-20 * ((x - 0.4) ** 2 + (y - 0.5) ** 2)),
                sigma_a=lambda x, y: 0.2 + 0.1 * x, sigma_s0=lambda x, y: 1.5,
                sigma_sm=lambda x, y, m: 0.7 ** m * (1 + 0.1 * y),
                filterfunction=configs.exp_filter(2, 5.0), f_position="substep",
                tfinal=1.5, t_plot=[0, 1.5], quiet=True)


def pt3d_p3():
    return configs.pointsource3d(n=8, n_mom=3, tfinal=1.5, std=0.2)


def box3d_bc1_p2_full():
    return dict(name="box3d", closure="P", n_mom=2, ax=[0, 1, 0, 1.2, 0, 0.8], n=[6, 5, 4], bc=[1, 0, 1],
                ic=lambda x, y, z: np.exp(-10 * ((x - .5) ** 2 + (y - .6) ** 2 + (z - .4) ** 2)),
                sigma_a=lambda x, y, z: 0.1 + 0.3 * x * z, sigma_s0=lambda x, y, z: 0.8 + 0.1 * y,
                sigma_sm=lambda x, y, z, m: 0.2 / (m + 1),
                source=lambda x, y, z, t: 0.5 * np.exp(-5 * ((x - .3) ** 2 + y ** 2)),
                filterfunction=lambda par, dt, k: np.exp(-dt * 3.0 * (k / 3.0) ** 2), f_position="full",
                tfinal=2.0, t_plot=[0, 2.0], quiet=True)


def spn_2d():
    return dict(name="spn2", closure="SP", n_mom=5, ax=[0, 2, 0, 2], n=[12, 10], bc=[1, 1],
                ic=lambda x, y: np.exp(-8 * ((x - 1) ** 2 + (y - 1) ** 2)),
                sigma_a=lambda x, y: 0.3, sigma_s0=lambda x, y: 0.7, tfinal=2.0, t_plot=[0, 2.0], quiet=True)


def spn_3d():
    return dict(name="spn3", closure="SP", n_mom=3, ax=[0, 1, 0, 1, 0, 1], n=[5, 6, 4], bc=[0, 0, 0],
                ic=lambda x, y, z: np.exp(-8 * ((x - .5) ** 2 + (y - .5) ** 2 + (z - .5) ** 2)),
                sigma_a=lambda x, y, z: 0.1, sigma_s0=lambda x, y, z: 1.0, tfinal=1.5, t_plot=[0, 1.5], quiet=True)


def one_d_p5():
    return dict(name="1d", closure="P", n_mom=5, ax=[-1, 1], n=[30], bc=[1],
                ic=lambda x: np.exp(-10 * x ** 2), sigma_a=lambda x: 0.1, sigma_s0=lambda x: 1.0,
                source=lambda x, t: 0.3 * (np.abs(x) < 0.3), tfinal=2.0, t_plot=[0, 2.0], quiet=True)


def boxes_td_source():
    """Time-dependent source of starmap_2d_ex_boxes.m:76-80 (P9 there; P3 here)."""
    def source(x, y, t):
        return (2 + np.sin(4 * np.pi * t) * np.exp(-t / 3)) * (
            ((1.75 < x) & (x <= 2.25) & (1.75 < y) & (y <= 2.25)) |
            ((2.75 < x) & (x <= 3.25) & (1.5 < y) & (y <= 2.50))).astype(np.float64)
    return dict(name="boxes", closure="P", n_mom=3, ax=[0, 5, 0, 5], n=[16, 16], bc=[1, 1],
                sigma_a=lambda x, y: 0.9, sigma_s0=lambda x, y: 0.1, source=source,
                tfinal=4.0, t_plot=[0, 4.0], quiet=True)


def td_sigma():
    return dict(name="tdsig", closure="P", n_mom=3, ax=[0, 1, 0, 1], n=[10, 9], bc=[0, 0],
                ic=lambda x, y: np.exp(-15 * ((x - .5) ** 2 + (y - .5) ** 2)),
                sigma_a=lambda x, y, t: 0.5 + t * np.cos(2 * np.pi * y), sigma_s0=lambda x, y: 1.0,
                tfinal=1.5, t_plot=[0, 1.5], quiet=True)


def parabolic_homog():
    """Parabolic time step (timestep 1) with homogeneous scalar materials, as
    starmap_2d_ex_homogeneous.m runs it (smaller grid and end time)."""
    return dict(name="parab", closure="P", n_mom=3, timestep=1, ax=[-1, 1, -1, 1], n=[14, 12], bc=[1, 1],
                ic=lambda x, y, k: np.exp(-((x ** 2 + y ** 2) / .25 ** 2) ** 2) * (k == 1),
                sigma_a=lambda x, y: 6.0, sigma_s0=lambda x, y: 6.0, tfinal=0.7, t_plot=[0, 0.7], quiet=True)


def parabolic_td():
    """Relative-stability parabolic step (timestep 2) with time-dependent
    absorption and a spatially varying scattering field: dt is searched every
    step."""
    return dict(name="parab_td", closure="P", n_mom=2, timestep=2, ax=[0, 1, 0, 1], n=[9, 11], bc=[0, 1],
                ic=lambda x, y: np.exp(-15 * ((x - .5) ** 2 + (y - .4) ** 2)),
                sigma_a=lambda x, y, t: 2.0 + np.sin(6 * t) + 0 * x, sigma_s0=lambda x, y: 4.0 + x * y,
                tfinal=0.35, t_plot=[0, 0.35], quiet=True)


ALL = {
    "lin_p7_periodic": lin_p7_periodic,
    "lattice_p5_substep": lattice_p5_substep,
    "lattice_p4_full": lattice_p4_full,
    "lattice_p6_nofilter": lattice_p6_nofilter,
    "odd_mixed_bc": odd_mixed_bc,
    "aniso_2d": aniso_2d,
    "pt3d_p3": pt3d_p3,
    "box3d_bc1_p2_full": box3d_bc1_p2_full,
    "spn_2d": spn_2d,
    "spn_3d": spn_3d,
    "one_d_p5": one_d_p5,
    "boxes_td_source": boxes_td_source,
    "td_sigma": td_sigma,
    "parabolic_homog": parabolic_homog,
    "parabolic_td": parabolic_td,
}
