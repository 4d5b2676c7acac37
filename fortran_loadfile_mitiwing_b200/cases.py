"""Input generators for the benchmark and parity cases: NACA 0012 contours,
motion tables in the motion_params.dat layout, run parameters, and the seeded
initial perturbation.

The reference reads its contour from boundary.dat (airfoil.f90:207-242): a
closed NACA 0012 of chord 1 with x in [-0.25, 0.75] (the pivot at x=0 is the
quarter chord), points uniform in x with one extra point a quarter step behind
the leading edge, closed trailing edge (thickness
coefficient -0.1036), first point = last point at the leading edge, upper
surface first. `naca0012(n_markers)` writes the same layout for any number of
markers. The motion columns follow apply_motion_row (mode.f90:161-171): per
wing angle, omega, omgac, sa, sau, saac, sb, sbv, sbac, with time t* = t U0/c
(the driver's time = (n-1)*scale*UU, main.f90:352), positions in chords,
velocities in units of U0, angle positive nose-up (airfoil.f90:261-263).
"""
import math

import numpy as np

from ._abi import LbmParams, LBM_DELTA_PESKIN4, PRECISIONS


def naca0012(n_markers, spacing="uniform-x"):
    """Closed NACA 0012 contour with n_markers segments (n_markers+1 points).

    spacing "uniform-x" is the reference file's layout; "cosine" clusters points
    at both ends (x = (1-cos b)/2). Returns (x, y) in chords, body frame.
    """
    if n_markers < 4 or n_markers % 2:
        raise ValueError("n_markers must be even and >= 4")
    m = n_markers // 2
    if spacing == "uniform-x":
        # the reference file's layout: x uniform with step h = 1/(m-1), plus one
        # point at h/4 behind the leading edge
        h = 1.0 / (m - 1)
        xs = np.concatenate([[0.0, 0.25 * h], h * np.arange(1, m)])
        xs[-1] = 1.0
    elif spacing == "cosine":
        xs = 0.5 * (1.0 - np.cos(np.linspace(0.0, math.pi, m + 1)))
    else:
        raise ValueError(spacing)
    yt = 0.6 * (0.2969 * np.sqrt(xs) - 0.1260 * xs - 0.3516 * xs**2 + 0.2843 * xs**3 - 0.1036 * xs**4)
    yt[0] = 0.0
    yt[-1] = 0.0
    x = np.concatenate([xs, xs[::-1][1:]]) - 0.25
    y = np.concatenate([yt, -yt[::-1][1:]])
    # the file holds 8 decimals (format 2f14.8); round so files and memory agree
    return np.round(x, 8), np.round(y, 8)


def plunge_pitch_table(n_steps, dt, n_wings=1, heave=0.0, pitch_deg=0.0, phase_deg=0.0, freq=0.0,
                       surge=0.0):
    """Motion table (rows, 1+9*n_wings), one row per time step t*=(i-1)*dt.

    sb = heave*sin(2 pi f t), angle = pitch*sin(2 pi f t + phase) (radians),
    with their first and second time derivatives in omega/omgac and sbv/sbac.
    """
    t = np.arange(n_steps, dtype=np.float64) * dt
    w = 2.0 * math.pi * freq
    th0 = math.radians(pitch_deg)
    ph = math.radians(phase_deg)
    cols = [t]
    for _ in range(n_wings):
        angle = th0 * np.sin(w * t + ph)
        omega = th0 * w * np.cos(w * t + ph)
        omgac = -th0 * w * w * np.sin(w * t + ph)
        sa = np.full_like(t, surge)
        sau = np.zeros_like(t)
        saac = np.zeros_like(t)
        sb = heave * np.sin(w * t)
        sbv = heave * w * np.cos(w * t)
        sbac = -heave * w * w * np.sin(w * t)
        cols += [angle, omega, omgac, sa, sau, saac, sb, sbv, sbac]
    return np.stack(cols, axis=1)


def make_params(nx, ny, chord_lu, pivot_node, uu, re, s=None, wings=1, markers=160,
                delta=LBM_DELTA_PESKIN4, precision="fp32"):
    """lbm_params for a lattice nx x ny with the pivot on 1-based node pivot_node."""
    p = LbmParams()
    p.nx, p.ny = nx, ny
    p.wing_count = wings
    p.points_per_wing = markers + 1 if wings > 0 else 0
    p.delta_kernel = delta
    p.precision = PRECISIONS[precision] if isinstance(precision, str) else precision
    p.scale = 1.0 / chord_lu
    p.ox = -(pivot_node[0] - 1) * p.scale
    p.oy = -(pivot_node[1] - 1) * p.scale
    p.uu = uu
    p.re = re
    if s is None:
        s = (0.0, 1.64, 1.54, 0.0, 1.9, 0.0, 1.9, 0.0, 0.0)   # s8, s9 <= 0: 1/tau
    for k in range(9):
        p.s[k] = s[k]
    p.xc = p.yc = p.xp = p.yp = 0.0
    p.mesh_max_scale = p.scale
    return p


def perturbation(nx, ny, amp=1.0e-4, seed=20261203):
    """Seeded uniform perturbation U(-amp, amp) for u and v, (nx, ny) Fortran order."""
    rng = np.random.default_rng(seed)
    du = rng.uniform(-amp, amp, size=nx * ny)
    dv = rng.uniform(-amp, amp, size=nx * ny)
    return du, dv


class Case:
    """A complete input set: params, one contour per wing, motion table, perturbation."""

    def __init__(self, name, params, contours, table, du=None, dv=None, n_steps=None):
        self.name = name
        self.params = params
        self.contours = contours
        self.table = np.ascontiguousarray(table, dtype=np.float64)
        self.du = du
        self.dv = dv
        self.n_steps = n_steps if n_steps is not None else table.shape[0]

    def with_precision(self, precision):
        import copy
        p = copy.copy(self.params)
        p.precision = PRECISIONS[precision] if isinstance(precision, str) else precision
        return Case(self.name, p, self.contours, self.table, self.du, self.dv, self.n_steps)


def plunge_case(nx=400, ny=200, chord=80, pivot=(100, 100), markers=160, n_steps=4000, re=100.0,
                uu=0.05, st=0.3, heave=0.25, precision="fp32", seed=20261203, amp=1.0e-4):
    """The plain 400x200 plunging NACA 0012 case: chord 80 lu, U0=0.05, Re=100,
    s=(0,1.64,1.54,0,1.9,0,1.9,1/tau,1/tau), 4-point delta, 160 markers,
    y = 0.25c sin(2 pi f t) with St = 2 f (0.25c)/U0 = 0.3, seeded 1e-4 perturbation."""
    p = make_params(nx, ny, chord, pivot, uu, re, markers=markers, precision=precision)
    x, y = naca0012(markers)
    freq = st / (2.0 * heave)
    table = plunge_pitch_table(n_steps, p.scale * uu, heave=heave, freq=freq)
    du, dv = perturbation(nx, ny, amp, seed) if amp > 0 else (None, None)
    return Case(f"plunge{nx}x{ny}", p, [(x, y)], table, du, dv, n_steps)


def heave_pitch_case(nx=4096, ny=2048, chord=512, pivot=(1025, 1025), markers=1024, n_steps=100000,
                     re=1000.0, uu=0.05, st=0.3, heave=0.5, pitch_deg=30.0, phase_deg=90.0,
                     precision="fp32", seed=20261203, amp=1.0e-4):
    """The single large 4096x2048 case: chord 512 lu, Re=1000, 1024 markers,
    y = 0.5c sin(2 pi f t), theta = 30 deg sin(2 pi f t + 90 deg) about the
    quarter chord, St = 2 f (0.5c)/U0 = 0.3."""
    p = make_params(nx, ny, chord, pivot, uu, re, markers=markers, precision=precision)
    x, y = naca0012(markers)
    freq = st / (2.0 * heave)
    table = plunge_pitch_table(n_steps, p.scale * uu, heave=heave, pitch_deg=pitch_deg,
                               phase_deg=phase_deg, freq=freq)
    du, dv = perturbation(nx, ny, amp, seed) if amp > 0 else (None, None)
    return Case(f"heavepitch{nx}x{ny}", p, [(x, y)], table, du, dv, n_steps)


def small_case(nx=96, ny=64, chord=24, pivot=(33, 33), markers=40, n_steps=200, re=100.0, uu=0.05,
               heave=0.25, pitch_deg=10.0, st=0.3, precision="fp32", wings=1, delta=LBM_DELTA_PESKIN4,
               amp=1.0e-4, seed=7):
    """A small case that the oracle steps in milliseconds, with heave and pitch."""
    p = make_params(nx, ny, chord, pivot, uu, re, markers=markers, precision=precision, wings=wings,
                    delta=delta)
    x, y = naca0012(markers)
    freq = st / (2.0 * heave) if heave > 0 else 0.5
    table = plunge_pitch_table(n_steps, p.scale * uu, n_wings=wings, heave=heave, pitch_deg=pitch_deg,
                               freq=freq)
    if wings == 2:
        # second wing: a tandem copy one chord downstream
        table[:, 1 + 9 + 3] = 1.5
    du, dv = perturbation(nx, ny, amp, seed) if amp > 0 else (None, None)
    return Case(f"small{nx}x{ny}", p, [(x, y)] * max(wings, 0), table, du, dv, n_steps)
