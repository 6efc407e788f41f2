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

    def tracks(self, begin, end):
        """The tracks [begin, end) with their hits (same detector)."""
        d = dict(self.__dict__)
        d.update(par=np.ascontiguousarray(self.par[:, begin:end]),
                 err=np.ascontiguousarray(self.err[:, begin:end]),
                 chg=np.ascontiguousarray(self.chg[begin:end]),
                 hit_pos=np.ascontiguousarray(self.hit_pos[:, :, begin:end]),
                 hit_err=np.ascontiguousarray(self.hit_err[:, :, begin:end]))
        return FitEvent(**d)


def gen_fit_event(n_tracks=20000, seed=0xC0FFEE, radii=None, pt_range=(0.5, 10.0),
                  eta_max=1.0, sig_rphi=0.01, sig_z=0.1, x_over_x0=0.01,
                  vtx_sigma_xy=0.01, vtx_sigma_z=5.0, r_start=1.0, align_rphi=None,
                  align_z=None, mat_scale=None):
    """Plain Kalman-fit toy MC: pT uniform, eta uniform in [-eta_max, eta_max],
    phi uniform, charge +-1, Gaussian vertex, one hit per cylinder layer with
    Gaussian r-phi / z smearing and a Highland multiple-scattering kick of
    `x_over_x0` radiation lengths (corrected for the crossing angle) at each
    layer. The initial state is the true state at radius r_start (default
    1 cm, outside the vertex spread); its covariance is a fixed diagonal.

    Misaligned detector (differentiable-fit workload): layer l is displaced
    by align_rphi[l] along the transverse tangent and align_z[l] in z, so the
    recorded hit (nominal geometry) is the true one moved back by those
    offsets; its material is mat_scale[l] times nominal (scattering kick)."""
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
        if align_rphi is not None:
            hpos[li, 0] += np.sin(pphi) * align_rphi[li]
            hpos[li, 1] -= np.cos(pphi) * align_rphi[li]
        if align_z is not None:
            hpos[li, 2] -= align_z[li]
        herr[li] = barrel_hit_errors(pphi, sig_rphi, sig_z)
        # Multiple scattering at the layer.
        p = hel.pt / np.sin(hel.theta)
        beta = p / np.sqrt(p * p + mpi * mpi)
        xl = x_over_x0 * (mat_scale[li] if mat_scale is not None else 1.0)
        t0 = highland(p, beta, xl * p / hel.pt)
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


def toy_material_grid_zr(radii, disks_z, x_over_x0=0.01, xi_per_x0=0.00217):
    """toy_material_grid with, in addition, `x_over_x0` radiation lengths on
    every disk at |z| in `disks_z` (the integer-cm z bins either side of it,
    all radii); the reference looks the grid up at bin int(|z|)."""
    rl, xi = toy_material_grid(radii, x_over_x0, xi_per_x0)
    for z in disks_z:
        for zb in (int(math.floor(abs(z))) - 1, int(math.floor(abs(z)))):
            if 0 <= zb < 300:
                rl[zb, :] = x_over_x0
                xi[zb, :] = x_over_x0 * xi_per_x0
    return rl, xi


def disk_hit_errors(phi, sig_rphi, sig_r, sig_z=0.01):
    """Hit covariance of a disk measurement smeared in r-phi and r at fixed
    z: the (x, y) block is R diag(sig_r^2, sig_rphi^2) R^T with R the
    rotation by phi."""
    n = phi.shape[0]
    e = np.zeros((6, n))
    sp, cp = np.sin(phi), np.cos(phi)
    a, b = sig_r ** 2, sig_rphi ** 2
    e[0] = a * cp * cp + b * sp * sp
    e[1] = (a - b) * sp * cp
    e[2] = a * sp * sp + b * cp * cp
    e[5] = np.full(n, sig_z ** 2)
    return e


def gen_fit_event_steered(n_tracks=20000, seed=0xF17E, radii=(4.0, 8.0),
                          disks_z=(35.0, 45.0, 55.0, 65.0, 75.0, 85.0, 95.0, 105.0),
                          pt_range=(1.0, 10.0), eta_range=(1.5, 2.0), sig_rphi=0.01,
                          sig_z=0.1, sig_r=0.1, x_over_x0=0.01, vtx_sigma_xy=0.01,
                          vtx_sigma_z=1.0, r_start=1.0):
    """Steered-fit toy MC (MkFitter::FitTracksSteered): forward tracks,
    |eta| uniform in eta_range with either sign, crossing the barrel
    cylinders `radii` first and then the disks at z = sign(eta) * disks_z
    (the defaults keep that order for every track). Step l is a barrel
    step for l < len(radii) and an endcap (z) step after: endcap_mask has
    the disk steps' bits. Smearing and multiple scattering as in
    gen_fit_event; disk hits are smeared in r-phi and r."""
    rng = np.random.default_rng(seed)
    radii = np.asarray(radii, dtype=np.float64)
    disks_z = np.asarray(disks_z, dtype=np.float64)
    n = n_tracks
    pt = rng.uniform(pt_range[0], pt_range[1], n)
    side = np.where(rng.random(n) < 0.5, -1.0, 1.0)
    eta = side * rng.uniform(eta_range[0], eta_range[1], n)
    phi = rng.uniform(-math.pi, math.pi, n)
    q = np.where(rng.random(n) < 0.5, -1, 1).astype(np.int32)
    vx = rng.normal(0.0, vtx_sigma_xy, n)
    vy = rng.normal(0.0, vtx_sigma_xy, n)
    vz = rng.normal(0.0, vtx_sigma_z, n)
    theta = 2.0 * np.arctan(np.exp(-eta))
    hel = Helix(vx, vy, vz, pt, phi, theta, q)
    s0 = hel.s_at_radius(np.full(n, r_start))
    x0, y0, z0, ph0 = hel.at(s0)
    hel.restart(np.ones(n, dtype=bool), x0, y0, z0, ph0, theta)
    par0 = np.stack([x0, y0, z0, 1.0 / pt, ph0, theta])
    cov = np.zeros((n, 6, 6))
    diag = np.stack([np.full(n, 0.1 ** 2), np.full(n, 0.1 ** 2), np.full(n, 1.0 ** 2),
                     (0.1 / pt) ** 2, np.full(n, 0.05 ** 2), np.full(n, 0.05 ** 2)], axis=1)
    for k in range(6):
        cov[:, k, k] = diag[:, k]

    nb, nd = radii.shape[0], disks_z.shape[0]
    hpos = np.zeros((nb + nd, 3, n))
    herr = np.zeros((nb + nd, 6, n))
    mpi = 0.140
    last_z = z0.copy()
    for li in range(nb + nd):
        if li < nb:
            s = hel.s_at_radius(np.full(n, radii[li]))
        else:
            s = hel.s_at_z(side * disks_z[li - nb])
        x, y, z, ph = hel.at(s)
        assert (np.abs(z) > np.abs(last_z)).all(), "crossings out of order"
        last_z = z
        pphi = np.arctan2(y, x)
        d = rng.normal(0.0, sig_rphi, n)
        if li < nb:
            hpos[li, 0] = x - np.sin(pphi) * d
            hpos[li, 1] = y + np.cos(pphi) * d
            hpos[li, 2] = z + rng.normal(0.0, sig_z, n)
            herr[li] = barrel_hit_errors(pphi, sig_rphi, sig_z)
            path = 1.0 / np.sin(hel.theta)                       # p / pT
        else:
            dr = rng.normal(0.0, sig_r, n)
            hpos[li, 0] = x - np.sin(pphi) * d + np.cos(pphi) * dr
            hpos[li, 1] = y + np.cos(pphi) * d + np.sin(pphi) * dr
            hpos[li, 2] = z
            herr[li] = disk_hit_errors(pphi, sig_rphi, sig_r)
            path = 1.0 / np.abs(np.cos(hel.theta))               # p / |pz|
        p = hel.pt / np.sin(hel.theta)
        beta = p / np.sqrt(p * p + mpi * mpi)
        t0 = highland(p, beta, x_over_x0 * path)
        th_new = hel.theta + rng.normal(0.0, 1.0, n) * t0
        ph_new = ph + rng.normal(0.0, 1.0, n) * t0 / np.sin(hel.theta)
        hel.restart(np.ones(n, dtype=bool), x, y, z, ph_new, th_new)

    rl, xi = toy_material_grid_zr(radii, disks_z, x_over_x0)
    endcap_mask = ((1 << (nb + nd)) - 1) & ~((1 << nb) - 1)
    return FitEvent(
        par=np.ascontiguousarray(par0, dtype=np.float32),
        err=np.ascontiguousarray(pack_sym(cov), dtype=np.float32),
        chg=q,
        hit_pos=np.ascontiguousarray(hpos, dtype=np.float32),
        hit_err=np.ascontiguousarray(herr, dtype=np.float32),
        radii=radii, disks_z=disks_z, endcap_mask=endcap_mask, rl_grid=rl, xi_grid=xi,
        seed=seed)


# =============================================================================
# CMS-2017 finding events
# =============================================================================

class CmsEvent:
    """Finding workload on the CMS-2017 geometry. Hits of all layers in one
    SoA buffer (layer l at [layer_begin[l], layer_begin[l+1])); seeds with up
    to 4 hits given as (layer, index within layer)."""

    def __init__(self, **kw):
        self.__dict__.update(kw)

    @property
    def n_seeds(self):
        return self.seed_chg.shape[0]

    @property
    def n_hits(self):
        return int(self.layer_begin[-1])


def _next_crossing(st, rs, is_barrel, zmin, zmax, rin, rout, hole, hmin, hmax, ptarget, done_mask):
    """For every live track, the smallest positive arc length to a layer
    surface it has not crossed yet and that is inside the layer's active
    extent. Barrel surfaces are cylinders r = propagate_to (outgoing side
    only), endcap surfaces planes z = propagate_to. Returns (s, layer) with
    s = inf where nothing is left before the apex."""
    n = st["x"].shape[0]
    L = is_barrel.shape[0]
    kap = st["kappa"][:, None]
    xc = st["x"] - np.sin(st["phi"]) / st["kappa"]
    yc = st["y"] + np.cos(st["phi"]) / st["kappa"]
    rho = 1.0 / np.abs(st["kappa"])
    d = np.hypot(xc, yc)
    alpha = np.arctan2(yc, xc)
    # psi: angle of the track point seen from the circle centre; dpsi/ds = kappa.
    psi0 = np.arctan2(st["y"] - yc, st["x"] - xc)
    period = 2 * np.pi * rho
    s_apex = np.mod((alpha - psi0) / st["kappa"], period)
    s = np.full((n, L), np.inf)
    # Barrel cylinders.
    rb = ptarget[None, :]
    c = (rb ** 2 - d[:, None] ** 2 - rho[:, None] ** 2) / (2 * d[:, None] * rho[:, None])
    ok = np.abs(c) <= 1.0
    ac = np.arccos(np.clip(c, -1, 1))
    for sgn in (1.0, -1.0):
        psi = alpha[:, None] + sgn * ac
        ss = np.mod((psi - psi0[:, None]) / kap, period[:, None])
        good = ok & is_barrel[None, :] & (ss > 1e-6) & (ss <= s_apex[:, None])
        s = np.where(good & (ss < s), ss, s)
    zc = st["z"][:, None] + s / np.tan(st["theta"])[:, None]
    s = np.where(is_barrel[None, :] & ((zc < zmin[None, :]) | (zc > zmax[None, :])), np.inf, s)
    # Endcap planes.
    se = (ptarget[None, :] - st["z"][:, None]) * np.tan(st["theta"])[:, None]
    good = (~is_barrel[None, :]) & (se > 1e-6) & (se <= s_apex[:, None])
    ph = st["phi"][:, None] + kap * se
    xe = st["x"][:, None] + (np.sin(ph) - np.sin(st["phi"])[:, None]) / kap
    ye = st["y"][:, None] - (np.cos(ph) - np.cos(st["phi"])[:, None]) / kap
    re = np.hypot(xe, ye)
    inside = (re > rin[None, :]) & (re < rout[None, :]) & ~(hole[None, :] & (re > hmin[None, :]) & (re < hmax[None, :]))
    s = np.where(good & inside, se, s)
    s = np.where(done_mask, np.inf, s)
    lay = np.argmin(s, axis=1)
    return s[np.arange(n), lay], lay


def gen_cms_event(n_tracks=800, seed=0xC0FFEE, geom=None, pt_range=(0.5, 50.0), eta_max=2.4,
                  noise_frac=0.01, noise_scale=None, vtx_sigma_xy=0.01, vtx_sigma_z=5.0,
                  r_start=1.0, overlap_prob=0.05, strip_len=10.0, seed_layers=None, seed_hits=3):
    """Synthetic CMS-2017 event: helices with pT log-uniform in pt_range,
    |eta| < eta_max, transported through the layer table with a Highland
    multiple-scattering kick from the reference material grid at each
    crossing; one hit per crossed layer (pixel: 0.003 cm in both measured
    directions; strip: 0.01 cm in r-phi, uniform along a strip of
    `strip_len` cm on the long axis) plus, with probability `overlap_prob`
    on strip layers, a second hit in the neighbouring module; noise hits at
    `noise_frac` of each layer's signal-hit count (times `noise_scale[l]`
    when given) uniform in the layer's extent. Seeds: the first `seed_hits`
    hits on seed layers (default the pixel layers; `seed_layers` a
    per-layer boolean mask) of every track that has them, with the true
    state at the last of them and a fixed diagonal covariance."""
    from .geometry import cms2017
    g = geom or cms2017()
    rng = np.random.default_rng(seed)
    n = n_tracks
    L = g.n_layers
    is_barrel = g.field("is_barrel") > 0.5
    zmin, zmax = g.field("zmin").astype(np.float64), g.field("zmax").astype(np.float64)
    rin, rout = g.field("rin").astype(np.float64), g.field("rout").astype(np.float64)
    hole = g.field("has_hole") > 0.5
    hmin, hmax = g.field("hole_min").astype(np.float64), g.field("hole_max").astype(np.float64)
    is_pix = g.field("is_pix") > 0.5
    is_stereo = g.field("is_stereo") > 0.5
    # Generation surfaces: the layer's nominal surface; stereo layers (which
    # share it with their mono partner) are placed 0.5 cm further out.
    ptarget = g.field("propagate_to").astype(np.float64)
    ptarget = ptarget + np.where(is_stereo, 0.5 * np.sign(np.where(is_barrel, 1.0, ptarget)), 0.0)

    pt = np.exp(rng.uniform(np.log(pt_range[0]), np.log(pt_range[1]), n))
    eta = rng.uniform(-eta_max, eta_max, n)
    phi = rng.uniform(-math.pi, math.pi, n)
    q = np.where(rng.random(n) < 0.5, -1, 1).astype(np.int32)
    vx = rng.normal(0, vtx_sigma_xy, n)
    vy = rng.normal(0, vtx_sigma_xy, n)
    vz = rng.normal(0, vtx_sigma_z, n)
    theta = 2.0 * np.arctan(np.exp(-eta))
    hel = Helix(vx, vy, vz, pt, phi, theta, q)
    s0 = hel.s_at_radius(np.full(n, r_start))
    x, y, z, ph = hel.at(s0)
    st = dict(x=x, y=y, z=z, phi=ph, theta=theta.copy(), pt=pt.copy(),
              kappa=-q / curvature_radius(pt))
    done = np.zeros((n, L), dtype=bool)
    alive = np.ones(n, dtype=bool)
    hits = []  # (track, layer, x, y, z, phi_dir, theta_dir, pt)
    mpi = 0.140
    for _ in range(4 * L):
        idx = np.nonzero(alive)[0]
        if idx.size == 0:
            break
        sub = {k: v[idx] for k, v in st.items()}
        s, lay = _next_crossing(sub, None, is_barrel, zmin, zmax, rin, rout, hole, hmin, hmax,
                                ptarget, done[idx])
        fin = np.isfinite(s)
        alive[idx[~fin]] = False
        idx, s, lay = idx[fin], s[fin], lay[fin]
        if idx.size == 0:
            break
        kap = st["kappa"][idx]
        ph1 = st["phi"][idx] + kap * s
        x1 = st["x"][idx] + (np.sin(ph1) - np.sin(st["phi"][idx])) / kap
        y1 = st["y"][idx] - (np.cos(ph1) - np.cos(st["phi"][idx])) / kap
        z1 = st["z"][idx] + s / np.tan(st["theta"][idx])
        done[idx, lay] = True
        hits.append(np.stack([idx, lay, x1, y1, z1, ph1, st["theta"][idx], st["pt"][idx]], axis=1))
        # Multiple scattering from the material grid at the crossing.
        r1 = np.hypot(x1, y1)
        zb = np.minimum((np.abs(z1) * 300 / 300.0).astype(np.int64), 299)
        rbn = np.minimum((r1 * 120 / 120.0).astype(np.int64), 119)
        radl = g.rl[zb, rbn].astype(np.float64)
        th = st["theta"][idx]
        p = st["pt"][idx] / np.sin(th)
        beta = p / np.sqrt(p * p + mpi * mpi)
        geo = np.where(is_barrel[lay], 1.0 / np.sin(th), 1.0 / np.abs(np.cos(th)))
        xx0 = np.maximum(radl * geo, 1e-9)
        t0 = np.where(radl > 0, highland(p, beta, xx0), 0.0)
        st["theta"][idx] = th + rng.normal(0, 1, idx.size) * t0
        st["phi"][idx] = ph1 + rng.normal(0, 1, idx.size) * t0 / np.sin(th)
        st["x"][idx], st["y"][idx], st["z"][idx] = x1, y1, z1
        # Stop tracks leaving the tracker volume.
        out = (np.abs(z1) > 290) | (r1 > 115)
        alive[idx[out]] = False

    H = np.concatenate(hits, axis=0) if hits else np.zeros((0, 8))
    trk = H[:, 0].astype(np.int64)
    lay = H[:, 1].astype(np.int64)
    # Order hits of each track along the trajectory (generation order).
    order = np.arange(H.shape[0])

    def smear(Hs, lay_s):
        m = Hs.shape[0]
        x0, y0, z0 = Hs[:, 2], Hs[:, 3], Hs[:, 4]
        pphi = np.arctan2(y0, x0)
        pix = is_pix[lay_s]
        brl = is_barrel[lay_s]
        stereo = is_stereo[lay_s]
        sig_t = np.where(pix, 0.003, 0.01)
        dt = rng.normal(0, 1, m) * sig_t
        # long axis: pixel Gaussian 0.003; strip uniform along the strip
        # (stereo strips: 0.1 cm Gaussian, a matched 2-D measurement).
        long_sig = np.where(pix, 0.003, np.where(stereo, 0.1, strip_len / math.sqrt(12.0)))
        dl = np.where(pix | stereo, rng.normal(0, 1, m) * long_sig,
                      rng.uniform(-0.5, 0.5, m) * strip_len)
        tx, ty = -np.sin(pphi), np.cos(pphi)
        hx = x0 + tx * dt
        hy = y0 + ty * dt
        hz = z0.copy()
        # barrel: long axis = z; endcap: long axis = radial.
        hz = np.where(brl, hz + dl, hz)
        hx = np.where(brl, hx, hx + np.cos(pphi) * dl)
        hy = np.where(brl, hy, hy + np.sin(pphi) * dl)
        e = np.zeros((6, m))
        st2 = sig_t ** 2
        ll2 = long_sig ** 2
        sp, cp = np.sin(pphi), np.cos(pphi)
        # barrel: transverse (r-phi) in xy, long in z.
        bxx, bxy, byy, bzz = st2 * sp * sp, -st2 * sp * cp, st2 * cp * cp, ll2
        # endcap: xy = R diag(radial=ll2, tangential=st2) R^T, zz tiny.
        exx = ll2 * cp * cp + st2 * sp * sp
        exy = (ll2 - st2) * sp * cp
        eyy = ll2 * sp * sp + st2 * cp * cp
        e[0] = np.where(brl, bxx, exx)
        e[1] = np.where(brl, bxy, exy)
        e[2] = np.where(brl, byy, eyy)
        e[5] = np.where(brl, bzz, 1e-6)
        return np.stack([hx, hy, hz]), e

    pos, err = smear(H, lay)
    # Module ids (12 bits): barrel 64 phi x 32 z segments, endcap 64 phi x 32 r rings.
    def module_id(px, py, pz, lay_s):
        pphi = np.arctan2(py, px)
        iphi = np.clip(((pphi + math.pi) / (2 * math.pi) * 64).astype(np.int64), 0, 63)
        brl = is_barrel[lay_s]
        fz = (pz - zmin[lay_s]) / np.maximum(zmax[lay_s] - zmin[lay_s], 1e-6)
        fr = (np.hypot(px, py) - rin[lay_s]) / np.maximum(rout[lay_s] - rin[lay_s], 1e-6)
        iq = np.clip((np.where(brl, fz, fr) * 32).astype(np.int64), 0, 31)
        return (iphi * 32 + iq).astype(np.int32)

    detid = module_id(H[:, 2], H[:, 3], H[:, 4], lay)
    mc = trk.astype(np.int32)

    # Overlap hits on strip layers: a second measurement in the neighbouring
    # module, 0.3 cm further out along the track.
    ov = (~is_pix[lay]) & (rng.random(H.shape[0]) < overlap_prob)
    if ov.any():
        Ho = H[ov].copy()
        kap = -np.sign(np.zeros(ov.sum()) + 1)  # placeholder, replaced below
        qtrk = q[trk[ov]].astype(np.float64)
        kap = -qtrk / curvature_radius(Ho[:, 7])
        ds = 0.3
        ph2 = Ho[:, 5] + kap * ds
        Ho[:, 2] = Ho[:, 2] + (np.sin(ph2) - np.sin(Ho[:, 5])) / kap
        Ho[:, 3] = Ho[:, 3] - (np.cos(ph2) - np.cos(Ho[:, 5])) / kap
        Ho[:, 4] = Ho[:, 4] + ds / np.tan(Ho[:, 6])
        lay_o = lay[ov]
        pos_o, err_o = smear(Ho, lay_o)
        det_o = ((detid[ov] + 32) % 2048).astype(np.int32)
        pos = np.concatenate([pos, pos_o], axis=1)
        err = np.concatenate([err, err_o], axis=1)
        lay = np.concatenate([lay, lay_o])
        detid = np.concatenate([detid, det_o])
        mc = np.concatenate([mc, trk[ov].astype(np.int32)])
        trk = np.concatenate([trk, trk[ov]])
        order = np.concatenate([order, np.full(ov.sum(), 1 << 40)])

    # Noise hits.
    n_sig = np.bincount(lay, minlength=L)
    scale = np.ones(L) if noise_scale is None else np.asarray(noise_scale, dtype=np.float64)
    n_noise = rng.poisson(noise_frac * n_sig * scale)
    nz_pos, nz_err, nz_lay, nz_det = [], [], [], []
    for l in range(L):
        k = int(n_noise[l])
        if k == 0:
            continue
        pphi = rng.uniform(-math.pi, math.pi, k)
        if is_barrel[l]:
            r = np.full(k, ptarget[l])
            zz = rng.uniform(zmin[l], zmax[l], k)
        else:
            r = rng.uniform(rin[l], rout[l], k)
            if hole[l]:
                r = np.where((r > hmin[l]) & (r < hmax[l]), rin[l] + 0.5 * (hmin[l] - rin[l]), r)
            zz = np.full(k, ptarget[l])
        Hn = np.zeros((k, 8))
        Hn[:, 2], Hn[:, 3], Hn[:, 4] = r * np.cos(pphi), r * np.sin(pphi), zz
        pn, en = smear(Hn, np.full(k, l))
        nz_pos.append(pn)
        nz_err.append(en)
        nz_lay.append(np.full(k, l))
        nz_det.append(module_id(Hn[:, 2], Hn[:, 3], Hn[:, 4], np.full(k, l)))
    if nz_pos:
        pos = np.concatenate([pos] + nz_pos, axis=1)
        err = np.concatenate([err] + nz_err, axis=1)
        lay = np.concatenate([lay] + nz_lay)
        detid = np.concatenate([detid] + nz_det).astype(np.int32)
        nn = sum(a.shape[0] for a in nz_lay)
        mc = np.concatenate([mc, np.full(nn, -1, np.int32)])
        trk = np.concatenate([trk, np.full(nn, -1)])
        order = np.concatenate([order, np.full(nn, 1 << 41)])

    m = lay.shape[0]
    # Strip charge per cm: mostly saturated (always passes the charge cut),
    # a fifth spread over [1700, 3600] so the cut is exercised.
    cpcm = np.where(is_pix[lay], -1,
                    np.where(rng.random(m) < 0.8, 4000, rng.integers(1700, 3600, m))).astype(np.int32)

    # Group by layer, random order within a layer.
    perm = np.lexsort((rng.random(m), lay))
    lay_sorted = lay[perm]
    layer_begin = np.zeros(L + 1, np.int32)
    layer_begin[1:] = np.cumsum(np.bincount(lay_sorted, minlength=L))
    inv = np.empty(m, np.int64)
    inv[perm] = np.arange(m)
    index_in_layer = inv - layer_begin[lay]

    # Seeds: first seed_hits hits on seed layers (generation order) of each track.
    seed_mask = is_pix if seed_layers is None else np.asarray(seed_layers, bool)
    sig_idx = np.nonzero((mc >= 0) & seed_mask[lay] & (order < (1 << 40)))[0]
    sig_idx = sig_idx[np.lexsort((order[sig_idx], trk[sig_idx]))]
    seeds = []
    t_prev, cnt = -1, 0
    first3 = {}
    for h in sig_idx:
        t = int(trk[h])
        if t != t_prev:
            t_prev, cnt = t, 0
        if cnt < seed_hits:
            first3.setdefault(t, []).append(h)
        cnt += 1
    seed_tracks = sorted(t for t, v in first3.items() if len(v) == seed_hits)
    ns = len(seed_tracks)
    spar = np.zeros((6, ns))
    serr = np.zeros((21, ns))
    schg = np.zeros(ns, np.int32)
    snh = np.full(ns, seed_hits, np.int32)
    shl = np.full((ns, max(4, seed_hits)), -1, np.int32)
    shi = np.full((ns, max(4, seed_hits)), -1, np.int32)
    for i, t in enumerate(seed_tracks):
        hs = first3[t]
        Hh = H[hs[-1]]  # true crossing of the last seed hit (signal hits precede overlaps)
        spar[:, i] = [Hh[2], Hh[3], Hh[4], 1.0 / Hh[7], Hh[5], Hh[6]]
        d = [0.01 ** 2, 0.01 ** 2, 0.01 ** 2, (0.05 / Hh[7]) ** 2, 0.005 ** 2, 0.005 ** 2]
        for k, (a, b) in enumerate(SYM6):
            if a == b:
                serr[k, i] = d[a]
        schg[i] = q[t]
        for k, h in enumerate(hs):
            shl[i, k] = lay[h]
            shi[i, k] = index_in_layer[h]
    return CmsEvent(
        n_layers=L, layer_begin=layer_begin,
        hit_pos=np.ascontiguousarray(pos[:, perm], np.float32),
        hit_err=np.ascontiguousarray(err[:, perm], np.float32),
        hit_detid=np.ascontiguousarray(detid[perm], np.int32),
        hit_cpcm=np.ascontiguousarray(cpcm[perm], np.int32),
        hit_mc=np.ascontiguousarray(mc[perm], np.int32),
        seed_par=np.ascontiguousarray(spar, np.float32),
        seed_err=np.ascontiguousarray(serr, np.float32),
        seed_chg=schg, seed_nhits=snh, seed_hit_layer=shl, seed_hit_index=shi,
        seed_mc=np.array(seed_tracks, np.int32), n_tracks=n, seed=seed,
        n_signal_hits=int((mc >= 0).sum()))


def density_ramp(n_layers, ratio=20.0):
    """Per-layer noise multipliers rising geometrically from 1 to `ratio`
    over the layer index (hit density varying ~ratio x across layers)."""
    return np.power(ratio, np.arange(n_layers) / max(n_layers - 1, 1))


def batch_event_sizes(n_events, mean, lo, hi, seed):
    """Poisson track counts per event, clipped to [lo, hi]."""
    rng = np.random.default_rng(seed)
    return np.clip(rng.poisson(mean, n_events), lo, hi).astype(int)


def gen_cms_event_args(args):
    """Picklable entry for process pools: gen_cms_event(**args)."""
    return gen_cms_event(**args)


def with_duplicate_seeds(ev, frac=0.25, seed=7, chain_frac=0.3):
    """Seeds of `ev` plus near-duplicates, as a seeding step with overlapping
    seeds gives them: a copy of a seed with small shifts of its position and
    direction (tens of microns, ~1e-3 rad), 1/pT within a few percent and a
    different third hit (the next hit of the same layer); some duplicates are
    duplicated again (chains), and all are inserted at random places in the
    seed order. Returns the seed arrays (par, err, chg, nhits, hit_layer,
    hit_index) and `src`, the original seed each entry derives from."""
    rng = np.random.default_rng(seed)
    ns = ev.n_seeds
    par = [ev.seed_par[:, i].astype(np.float64) for i in range(ns)]
    err = [ev.seed_err[:, i] for i in range(ns)]
    chg = list(ev.seed_chg)
    nh = list(ev.seed_nhits)
    hl = [ev.seed_hit_layer[i].copy() for i in range(ns)]
    hi = [ev.seed_hit_index[i].copy() for i in range(ns)]
    src = list(range(ns))
    lb = ev.layer_begin

    def dup(i):
        p = par[i].copy()
        p[0:3] += rng.normal(0.0, 0.003, 3)
        p[3] *= 1.0 + rng.normal(0.0, 0.02)
        p[4] += rng.normal(0.0, 0.001)
        p[5] += rng.normal(0.0, 0.001)
        h_l, h_i = hl[i].copy(), hi[i].copy()
        k = nh[i] - 1
        if k >= 0 and rng.random() < 0.7:
            n_lay = lb[h_l[k] + 1] - lb[h_l[k]]
            h_i[k] = (h_i[k] + 1) % max(n_lay, 1)
        par.append(p)
        err.append(err[i])
        chg.append(chg[i])
        nh.append(nh[i])
        hl.append(h_l)
        hi.append(h_i)
        src.append(src[i])
        return len(par) - 1

    picks = rng.choice(ns, size=int(frac * ns), replace=False) if ns else []
    for i in picks:
        j = dup(int(i))
        if rng.random() < chain_frac:
            dup(j)
    order = rng.permutation(len(par))
    sel = lambda a: [a[k] for k in order]  # noqa: E731
    if not par:
        w = ev.seed_hit_layer.shape[1] if ev.seed_hit_layer.ndim == 2 else 4
        z = lambda *shape: np.zeros(shape, np.int32)  # noqa: E731
        return dict(par=np.zeros((6, 0), np.float32), err=np.zeros((21, 0), np.float32),
                    chg=z(0), nhits=z(0), hit_layer=z(0, w), hit_index=z(0, w), src=z(0))
    return dict(
        par=np.ascontiguousarray(np.array(sel(par)).T, np.float32),
        err=np.ascontiguousarray(np.array(sel(err)).T, np.float32),
        chg=np.array(sel(chg), np.int32), nhits=np.array(sel(nh), np.int32),
        hit_layer=np.ascontiguousarray(np.array(sel(hl)), np.int32),
        hit_index=np.ascontiguousarray(np.array(sel(hi)), np.int32),
        src=np.array(sel(src), np.int32))


def without_first_seed_hit(ev):
    """The event with every seed's innermost hit taken out of the seed
    (three-hit seeds become hit pairs): the backward search then has that
    layer to find again, and hit-count cuts meet seeds of two hits."""
    d = dict(ev.__dict__)
    hl, hi = ev.seed_hit_layer.copy(), ev.seed_hit_index.copy()
    hl[:, :-1], hi[:, :-1] = ev.seed_hit_layer[:, 1:], ev.seed_hit_index[:, 1:]
    hl[:, -1] = hi[:, -1] = -1
    d.update(seed_hit_layer=hl, seed_hit_index=hi, seed_nhits=ev.seed_nhits - 1)
    return CmsEvent(**d)


def thinned(ev, frac, seed):
    """The event with a fraction `frac` of its non-pixel hits removed (an
    inefficient strip tracker): candidates come out short and with holes.
    Seeds keep their pixel hits and indices."""
    from .geometry import cms2017
    rng = np.random.default_rng(seed)
    is_pix = cms2017().field("is_pix") > 0.5
    lb = np.asarray(ev.layer_begin)
    keep = np.ones(ev.n_hits, bool)
    for lyr in range(ev.n_layers):
        if not is_pix[lyr]:
            keep[lb[lyr]:lb[lyr + 1]] = rng.random(lb[lyr + 1] - lb[lyr]) >= frac
    counts = [int(keep[lb[i]:lb[i + 1]].sum()) for i in range(ev.n_layers)]
    d = dict(ev.__dict__)
    d["layer_begin"] = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    for k in ("hit_pos", "hit_err"):
        d[k] = np.ascontiguousarray(getattr(ev, k)[:, keep])
    for k in ("hit_detid", "hit_cpcm", "hit_mc"):
        d[k] = np.ascontiguousarray(getattr(ev, k)[keep])
    return CmsEvent(**d)
