"""Seeded synthetic event generators (FP64 numpy).

The reference's toy-MC simulator is not part of the reference snapshot, so
these generators produce the inputs for every workload from a recorded seed.
They are input synthesis, not the algorithm under test: the same arrays feed
the GPU path and the reference CPU path.

Conventions (reference Config.h / Track.h):
  * track parameters in CCS coordinates: x, y, z [cm], 1/pT [1/GeV], phi, theta
  * a positive charge curls clockwise in +Bz; the transverse radius of
    curvature is R = 100 pT / (0.299792458 B) cm
  * B = 3.8112 T (the reference's Config::Bfield), used for generation and
    fitting alike.
"""
import math

import numpy as np

SOL = 0.299792458
BFIELD = 3.8112

# Index tables of the packed lower-triangle symmetric storage.
SYM6 = [(i, j) for i in range(6) for j in range(i + 1)]
SYM3 = [(i, j) for i in range(3) for j in range(i + 1)]


def curvature_radius(pt, b=BFIELD):
    return 100.0 * pt / (SOL * b)


class Helix:
    """Vectorised exact helix in a uniform Bz field, parameterised by the
    transverse arc length s travelled from a reference point."""

    def __init__(self, x, y, z, pt, phi, theta, q, b=BFIELD):
        self.x0, self.y0, self.z0 = x.copy(), y.copy(), z.copy()
        self.pt, self.phi0, self.theta = pt.copy(), phi.copy(), theta.copy()
        self.q = q.astype(np.float64)
        self.kappa = -self.q / curvature_radius(pt, b)  # dphi/ds

    def at(self, s):
        ph = self.phi0 + self.kappa * s
        x = self.x0 + (np.sin(ph) - np.sin(self.phi0)) / self.kappa
        y = self.y0 - (np.cos(ph) - np.cos(self.phi0)) / self.kappa
        z = self.z0 + s / np.tan(self.theta)
        return x, y, z, ph

    def s_at_radius(self, r, iters=8):
        """Smallest s >= 0 with rho(s) = r, by Newton iteration from the line
        estimate (the generators only ask for outward crossings well below
        the apex, where rho(s) is monotonic; converged to ~1e-12 cm)."""
        sp0, cp0 = np.sin(self.phi0), np.cos(self.phi0)
        ik = 1.0 / self.kappa
        r0 = np.hypot(self.x0, self.y0)
        s = np.maximum(r - r0, 0.0)
        for _ in range(iters):
            ph = self.phi0 + self.kappa * s
            sp, cp = np.sin(ph), np.cos(ph)
            x = self.x0 + (sp - sp0) * ik
            y = self.y0 - (cp - cp0) * ik
            rho = np.hypot(x, y)
            drho = (x * cp + y * sp) / np.maximum(rho, 1e-12)
            s = s - (rho - r) / np.where(np.abs(drho) > 1e-6, drho, 1e-6)
        return s

    def s_at_z(self, z):
        return (z - self.z0) * np.tan(self.theta)

    def restart(self, mask, x, y, z, phi, theta, pt=None):
        self.x0[mask], self.y0[mask], self.z0[mask] = x[mask], y[mask], z[mask]
        self.phi0[mask], self.theta[mask] = phi[mask], theta[mask]
        if pt is not None:
            self.pt[mask] = pt[mask]
            self.kappa[mask] = -self.q[mask] / curvature_radius(pt[mask])


def highland(p, beta, x_over_x0):
    """PDG multiple-scattering angle (plane projection)."""
    return 0.0136 / (beta * p) * np.sqrt(x_over_x0) * (1.0 + 0.038 * np.log(x_over_x0))


def pack_sym(mat):
    """(n, d, d) -> (d(d+1)/2, n) packed lower triangle, lane fastest."""
    d = mat.shape[-1]
    idx = SYM6 if d == 6 else SYM3
    return np.stack([mat[:, i, j] for (i, j) in idx], axis=0)


def barrel_hit_errors(phi, sig_rphi, sig_z):
    """Hit covariance of a barrel measurement smeared in r-phi and z:
    xx = s^2 sin^2(phi), yy = s^2 cos^2(phi), xy = -s^2 sin cos, zz = sz^2."""
    n = phi.shape[0]
    e = np.zeros((6, n))
    s2 = sig_rphi ** 2
    sp, cp = np.sin(phi), np.cos(phi)
    e[0] = s2 * sp * sp
    e[1] = -s2 * sp * cp
    e[2] = s2 * cp * cp
    e[5] = np.broadcast_to(np.asarray(sig_z, dtype=np.float64) ** 2, (n,))
    return e


def toy_material_grid(radii, x_over_x0=0.01, xi_per_x0=0.00217):
    """(z, r) material grid with `x_over_x0` radiation lengths at each given
    radius (the integer-cm r bins either side of it), zero elsewhere. The
    reference looks the grid up at bin int(r) (MaterialEffects.h:8-11)."""
    rl = np.zeros((300, 120), dtype=np.float32)
    xi = np.zeros((300, 120), dtype=np.float32)
    for r in radii:
        for rb in (int(math.floor(r)) - 1, int(math.floor(r))):
            if 0 <= rb < 120:
                rl[:, rb] = x_over_x0
                xi[:, rb] = x_over_x0 * xi_per_x0
    return rl, xi


class FitEvent:
    """Toy-MC fit workload: tracks with one hit on each of n_layers barrel
    cylinders. Arrays are lane-fastest SoA (float32 / int32)."""

    def __init__(self, **kw):
        self.__dict__.update(kw)

    @property
    def n(self):
        return self.chg.shape[0]


def gen_fit_event(n_tracks=20000, seed=0xC0FFEE, radii=None, pt_range=(0.5, 10.0),
                  eta_max=1.0, sig_rphi=0.01, sig_z=0.1, x_over_x0=0.01,
                  vtx_sigma_xy=0.01, vtx_sigma_z=5.0, r_start=1.0):
    """Plain Kalman-fit toy MC: pT uniform, eta uniform in [-eta_max, eta_max],
    phi uniform, charge +-1, Gaussian vertex, one hit per cylinder layer with
    Gaussian r-phi / z smearing and a Highland multiple-scattering kick of
    `x_over_x0` radiation lengths (corrected for the crossing angle) at each
    layer. The initial state is the true state at radius r_start (default
    1 cm, outside the vertex spread); its covariance is a fixed diagonal."""
    rng = np.random.default_rng(seed)
    if radii is None:
        radii = [4.0 * (i + 1) for i in range(10)]
    radii = np.asarray(radii, dtype=np.float64)
    n = n_tracks
    pt = rng.uniform(pt_range[0], pt_range[1], n)
    eta = rng.uniform(-eta_max, eta_max, n)
    phi = rng.uniform(-math.pi, math.pi, n)
    q = np.where(rng.random(n) < 0.5, -1, 1).astype(np.int32)
    vx = rng.normal(0.0, vtx_sigma_xy, n)
    vy = rng.normal(0.0, vtx_sigma_xy, n)
    vz = rng.normal(0.0, vtx_sigma_z, n)
    theta = 2.0 * np.arctan(np.exp(-eta))

    hel = Helix(vx, vy, vz, pt, phi, theta, q)
    # The fit starts from the true state at r_start: the reference's
    # iterative propagation flags tracks whose position and transverse
    # momentum point apart (mkFit/PropagationMPlex.icc:84-90), which is half
    # of all tracks when starting at a vertex smeared by ~0.01 cm.
    if r_start > 0:
        s0 = hel.s_at_radius(np.full(n, r_start))
        x0, y0, z0, ph0 = hel.at(s0)
    else:
        x0, y0, z0, ph0 = vx, vy, vz, phi
    hel.restart(np.ones(n, dtype=bool), x0, y0, z0, ph0, theta)
    par0 = np.stack([x0, y0, z0, 1.0 / pt, ph0, theta])
    cov = np.zeros((n, 6, 6))
    diag = np.stack([np.full(n, 0.1 ** 2), np.full(n, 0.1 ** 2), np.full(n, 1.0 ** 2),
                     (0.1 / pt) ** 2, np.full(n, 0.05 ** 2), np.full(n, 0.05 ** 2)], axis=1)
    for k in range(6):
        cov[:, k, k] = diag[:, k]

    nl = radii.shape[0]
    hpos = np.zeros((nl, 3, n))
    herr = np.zeros((nl, 6, n))
    mpi = 0.140
    for li, r in enumerate(radii):
        s = hel.s_at_radius(np.full(n, r))
        x, y, z, ph = hel.at(s)
        # Smear: tangential (r-phi) and longitudinal (z) Gaussian offsets.
        pphi = np.arctan2(y, x)
        d = rng.normal(0.0, sig_rphi, n)
        hpos[li, 0] = x - np.sin(pphi) * d
        hpos[li, 1] = y + np.cos(pphi) * d
        hpos[li, 2] = z + rng.normal(0.0, sig_z, n)
        herr[li] = barrel_hit_errors(pphi, sig_rphi, sig_z)
        # Multiple scattering at the layer.
        p = hel.pt / np.sin(hel.theta)
        beta = p / np.sqrt(p * p + mpi * mpi)
        t0 = highland(p, beta, x_over_x0 * p / hel.pt)
        th_new = hel.theta + rng.normal(0.0, 1.0, n) * t0
        ph_new = ph + rng.normal(0.0, 1.0, n) * t0 / np.sin(hel.theta)
        mask = np.ones(n, dtype=bool)
        hel.restart(mask, x, y, z, ph_new, th_new)

    rl, xi = toy_material_grid(radii, x_over_x0)
    return FitEvent(
        par=np.ascontiguousarray(par0, dtype=np.float32),
        err=np.ascontiguousarray(pack_sym(cov), dtype=np.float32),
        chg=q,
        hit_pos=np.ascontiguousarray(hpos, dtype=np.float32),
        hit_err=np.ascontiguousarray(herr, dtype=np.float32),
        radii=radii, rl_grid=rl, xi_grid=xi, seed=seed)
