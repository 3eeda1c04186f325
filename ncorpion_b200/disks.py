"""Seeded synthetic planetary disks in NcorpiON's body layout.

A body is the 8-double record of ``struct moonlet`` (``src/structure.h:74-84``):
``x, y, z, vx, vy, vz, mass, radius``.  Bodies orbit a central mass ``M = 1``
(``R_unit = M_unit = 1``) with ``G = 1``; orbital elements are drawn with
``numpy.random.default_rng(seed)`` and converted to cartesian coordinates with
the usual two-body (Kepler) formulae, using ``mu = G*(M + m)`` as the
reference's ``init()`` does (``src/structure.c:341-364``).

The disks are the five workloads the hot path is measured on:

* ``bf_collide``   N=2,000 equal masses (total 1e-3), R=2e-3, a~U[0.8,1.2]
* ``gravity``      N=65,536, masses log-uniform over [1e-9,1e-6], R=1e-5
* ``mesh``         N=1,048,576, a~U[0.5,2.0], dN/dR ~ R^-3.5 over [1e-5,1e-3]
* ``adjoint``      N=16,384, same law as ``gravity``
* ``fragment``     N=262,144, a~U[0.9,1.1], e,i Rayleigh 0.02, R~U[2e-4,5e-4]

``write_init_txt`` writes the reference's cartesian ``init.txt`` (8 columns
per line, read back with ``fscanf("%lf")`` in ``src/structure.c:1115-1145``);
17 significant digits make the text round trip exact.
"""
from __future__ import annotations

import numpy as np

G_DEFAULT = 1.0
M_CENTRAL = 1.0


def kepler_to_cartesian(a, e, inc, nu, omega, Omega, mu):
    """Cartesian position and velocity from (a, e, i, true anomaly, arg. of
    periapsis, longitude of node) for gravitational parameter ``mu``.
    All arguments are numpy arrays (or scalars) of float64."""
    p = a * (1.0 - e * e)
    r = p / (1.0 + e * np.cos(nu))
    cn, sn = np.cos(nu), np.sin(nu)
    # position / velocity in the orbital plane
    xo, yo = r * cn, r * sn
    sq = np.sqrt(mu / p)
    vxo, vyo = -sq * sn, sq * (e + cn)
    co, so = np.cos(omega), np.sin(omega)
    cO, sO = np.cos(Omega), np.sin(Omega)
    ci, si = np.cos(inc), np.sin(inc)
    # rotation Rz(Omega) Rx(i) Rz(omega)
    r11 = cO * co - sO * so * ci
    r12 = -cO * so - sO * co * ci
    r21 = sO * co + cO * so * ci
    r22 = -sO * so + cO * co * ci
    r31 = so * si
    r32 = co * si
    x = r11 * xo + r12 * yo
    y = r21 * xo + r22 * yo
    z = r31 * xo + r32 * yo
    vx = r11 * vxo + r12 * vyo
    vy = r21 * vxo + r22 * vyo
    vz = r31 * vxo + r32 * vyo
    return x, y, z, vx, vy, vz


def _assemble(rng, n, a_lo, a_hi, sig_e, sig_i, mass, radius, G=G_DEFAULT):
    a = rng.uniform(a_lo, a_hi, n)
    e = np.minimum(rng.rayleigh(sig_e, n), 0.9)
    inc = rng.rayleigh(sig_i, n)
    nu = rng.uniform(0.0, 2.0 * np.pi, n)
    om = rng.uniform(0.0, 2.0 * np.pi, n)
    Om = rng.uniform(0.0, 2.0 * np.pi, n)
    mu = G * (M_CENTRAL + mass)
    x, y, z, vx, vy, vz = kepler_to_cartesian(a, e, inc, nu, om, Om, mu)
    b = np.empty((n, 8), dtype=np.float64)
    b[:, 0], b[:, 1], b[:, 2] = x, y, z
    b[:, 3], b[:, 4], b[:, 5] = vx, vy, vz
    b[:, 6] = mass
    b[:, 7] = radius
    return b


def bf_collide_disk(n=2000, seed=0):
    """Brute-force collisional disk: equal masses summing to 1e-3, R=2e-3."""
    rng = np.random.default_rng(seed)
    mass = np.full(n, 1e-3 / n)
    radius = np.full(n, 2e-3)
    return _assemble(rng, n, 0.8, 1.2, 0.01, 0.005, mass, radius)


def gravity_disk(n=65536, seed=0, radius=1e-5):
    """Gravity-only disk: log-uniform masses over [1e-9, 1e-6], all R equal."""
    rng = np.random.default_rng(seed)
    mass = 10.0 ** rng.uniform(-9.0, -6.0, n)
    rad = np.full(n, radius)
    return _assemble(rng, n, 0.8, 1.2, 0.01, 0.005, mass, rad)


def powerlaw_radii(rng, n, r_lo, r_hi, q=3.5):
    """Inverse-CDF draw of dN/dR ~ R^-q over [r_lo, r_hi]."""
    u = rng.uniform(0.0, 1.0, n)
    k = 1.0 - q
    return (r_lo ** k + u * (r_hi ** k - r_lo ** k)) ** (1.0 / k)


def mesh_disk(n=1 << 20, seed=0, density=3.0):
    """Mesh collisional disk: a~U[0.5,2], R power law -3.5 over [1e-5,1e-3],
    constant density (mass = 4/3 pi rho R^3)."""
    rng = np.random.default_rng(seed)
    rad = powerlaw_radii(rng, n, 1e-5, 1e-3)
    mass = 4.0 / 3.0 * np.pi * density * rad ** 3
    return _assemble(rng, n, 0.5, 2.0, 0.01, 0.005, mass, rad)


def fragment_disk(n=262144, seed=0, density=3.0):
    """Fragmenting disk: a~U[0.9,1.1], e,i Rayleigh 0.02, R~U[2e-4,5e-4]."""
    rng = np.random.default_rng(seed)
    rad = rng.uniform(2e-4, 5e-4, n)
    mass = 4.0 / 3.0 * np.pi * density * rad ** 3
    return _assemble(rng, n, 0.9, 1.1, 0.02, 0.02, mass, rad)


def frag_test_disk(n=4000, seed=0, density=3.0):
    """Crowded, hot ring for the fragmentation parity cases: a~U[0.99,1.01],
    e,i Rayleigh 0.04, 60% of the radii U[1.5e-3,4e-3] and 40% U[1e-4,5e-4]
    (constant density).  One collision sweep with dt = 0.02 holds impacts of
    every outcome: merger, super-catastrophic, partial and full fragmentation."""
    rng = np.random.default_rng(seed)
    rad = rng.uniform(1.5e-3, 4e-3, n)
    small = rng.random(n) < 0.4
    rad[small] = rng.uniform(1e-4, 5e-4, int(small.sum()))
    mass = 4.0 / 3.0 * np.pi * density * rad ** 3
    return _assemble(rng, n, 0.99, 1.01, 0.04, 0.04, mass, rad)


def adjoint_disk(n=16384, seed=0, radius=1e-2):
    """Differentiable gravity-only disk: the law of ``gravity_disk`` with
    R = 1e-2, so that the softening length 0.5 (R_k + R_p) = 1e-2 (about the
    mean spacing) keeps every encounter smooth at dt = 1e-3.  With R = 1e-5 (the force-accuracy disk)
    bodies of up to 1e-6 central masses bind on orbits far shorter than dt, the
    1,000-step map is chaotic (gradient norms reach 1e22) and no finite
    difference with h = 1e-6 is in its linear regime."""
    return gravity_disk(n, seed, radius=radius)


def reduce_to_com(bodies, cm=None, G=G_DEFAULT):
    """Subtract the barycentre (central mass included) from positions and
    velocities, in the reference's summation order (``total_momentum``,
    ``src/structure.c:1193-1227``).  Returns (bodies, cm) as new arrays."""
    b = bodies.copy()
    c = np.array([0, 0, 0, 0, 0, 0, M_CENTRAL, 1.0]) if cm is None else cm.copy()
    M = c[6]
    mom = c[:6] * M
    m = b[:, 6]
    # sequential sums, like the reference loop
    for j in range(6):
        s = mom[j]
        col = m * b[:, j]
        for v in col:
            s += v
        mom[j] = s
    Mt = M
    for v in m:
        Mt += v
    com = mom / Mt
    b[:, :6] -= com
    c[:6] -= com
    return b, c


def write_init_txt(path, bodies):
    """Write ``init.txt`` in the reference's cartesian format (one body per
    line: x y z vx vy vz mass radius)."""
    np.savetxt(path, bodies, fmt="%.17g")
