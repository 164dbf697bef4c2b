"""Seeded synthetic scenarios (DATA objects) for tests and benchmarks.

The reference builds its inputs with Octave scripts that cannot run here
(data/*/*.m).  These generators restate their arithmetic with numpy:

* :func:`bench_slab`   -- data/performance/scaling.m:61-124 (the shipped
  DATA_bench_<N>.json fixtures);
* :func:`well_balance` -- data/well_balance/well_balance.m:1-234 (lake at
  rest over a Gaussian bump);
* :func:`conservation_bump` -- data/conservation_test/conservation_test.m;
* :func:`dam_break_flat`, :func:`mudflow`, :func:`ensemble_member`,
  :func:`serving_request` -- the workloads of the benchmark configurations
  (flat dam break 64x64 / 4096 particles; 2048^2 mudflow with ~4.0M
  particles; ensemble and serving members).

Particle order follows Octave's ``meshgrid(...)(:)``: y varies fastest.
Node arrays are in quadgrid order, node (r, c) at r + c*(Ney+1).
"""
from __future__ import annotations

import math

import numpy as np

from .data import DATA

DEFAULT_SEED = 12345


def _meshgrid_colmajor(xv: np.ndarray, yv: np.ndarray):
    """[X, Y] = meshgrid(xv, yv); returns X(:), Y(:) (column-major, y fastest)."""
    X, Y = np.meshgrid(xv, yv)  # shape (len(yv), len(xv))
    return X.reshape(-1, order="F"), Y.reshape(-1, order="F")


def _octave_range(base: float, inc: float, limit: float) -> np.ndarray:
    """Octave ``base:inc:limit`` (elements base + i*inc)."""
    n = int(math.floor((limit - base) / inc * (1 + 1e-15) + 1e-10)) + 1
    return base + np.arange(n, dtype=np.float64) * inc


def _octave_linspace(a: float, b: float, n: int) -> np.ndarray:
    """Octave ``linspace(a, b, n)``: a + i*delta, last element exactly b."""
    delta = (b - a) / (n - 1)
    v = a + np.arange(n, dtype=np.float64) * delta
    v[-1] = b
    return v


def _gradient(Zg: np.ndarray, hx: float, hy: float):
    """Octave ``[gx, gy] = gradient(Z, hx, hy)`` for Z of shape (ny, nx)."""
    gx = np.gradient(Zg, hx, axis=1, edge_order=1)
    gy = np.gradient(Zg, hy, axis=0, edge_order=1)
    return gx, gy


def _base_scalars(**kw) -> dict:
    s = {
        "Nex": 1, "Ney": 1, "hx": 1.0, "hy": 1.0, "rho": 1000.0, "g": 9.81,
        "T": 1.0, "xi": 200.0, "mu": 50.0, "phi": 20.0, "tauy": 30.0,
        "BINGHAM_ON": 0.0, "FRICTION_ON": 0.0, "CFL": 0.2, "BC_FLAG": 1,
        "MERGE_SPLIT_ON": 0, "eq_level": 0.0, "DT_FIXED": 0.0, "NSTEPS": 0,
        "ms_alpha": 0.9, "ms_beta": 0.30, "ms_split_hp_min": 0.0,
        "ms_shear_split": 1e30, "ms_hp_min": 0.05, "ms_max_dv": 0.01,
        "ms_min_level": -2, "ms_max_level": 2, "ms_min_particles_per_cell": 2,
        "ms_call_interval": 10, "ms_max_ops": 1e9, "ms_pair_dist": 0.0,
        "ms_variant": 0, "ms_stretch_thresh": 1e7,
    }
    s.update(kw)
    return s


def _particles(xp, yp, hp, Ap, rho, vpx=None, vpy=None) -> dict:
    n = xp.shape[0]
    Vp = Ap * hp
    Mp = rho * Vp
    z = np.zeros(n)
    vx = z.copy() if vpx is None else np.asarray(vpx, dtype=np.float64)
    vy = z.copy() if vpy is None else np.asarray(vpy, dtype=np.float64)
    return {"x": xp.astype(np.float64), "y": yp.astype(np.float64), "Mp": Mp,
            "Ap": Ap.astype(np.float64), "vpx": vx, "vpy": vy,
            "hp": hp.astype(np.float64), "mom_px": vx * Mp, "mom_py": vy * Mp,
            "Vp": Vp}


# ---------------------------------------------------------------------------
# data/performance/scaling.m:61-124
# ---------------------------------------------------------------------------
def bench_slab(N: int, dt_fixed: float = 1e-3, nsteps: int = 100) -> DATA:
    g, rho, xi, mu, phi, tauy = 9.81, 1200.0, 200.0, 2000.0, 20.0, 30.0
    hx = hy = 1.0
    s = 0.5
    slope = math.tan(2 * math.pi / 180)
    h0 = 5.0
    ncell = int(np.round(math.sqrt(N) / 2))
    Nex = Ney = ncell
    Lx, Ly = Nex * hx, Ney * hy
    x = _octave_linspace(0.0, Lx, Nex + 1)
    y = _octave_linspace(0.0, Ly, Ney + 1)
    X, Y = np.meshgrid(x, y)
    Zz = 100.0 - slope * X
    gx, gy = _gradient(Zz, hx, hy)
    m = 1.0
    xp = _octave_range(m + s / 2, s, Lx - m)
    yp = _octave_range(m + s / 2, s, Ly - m)
    xp, yp = _meshgrid_colmajor(xp, yp)
    n = xp.shape[0]
    hp = h0 * np.ones(n)
    Ap = (s * s) * np.ones(n)
    arrays = _particles(xp, yp, hp, Ap, rho)
    arrays.update({"Z": Zz.reshape(-1, order="F"), "dZdx": gx.reshape(-1, order="F"),
                   "dZdy": gy.reshape(-1, order="F")})
    sc = _base_scalars(Nex=Nex, Ney=Ney, hx=hx, hy=hy, rho=rho, g=g, T=20.0, xi=xi,
                       mu=mu, phi=phi, tauy=tauy, BINGHAM_ON=1.0, FRICTION_ON=1.0,
                       CFL=0.2, BC_FLAG=1, MERGE_SPLIT_ON=1, eq_level=0.0,
                       DT_FIXED=dt_fixed, NSTEPS=nsteps)
    return DATA(arrays, sc)


# ---------------------------------------------------------------------------
# data/well_balance/well_balance.m (lake at rest, eq_level 10)
# ---------------------------------------------------------------------------
def _interp2_linear(xv, yv, F, xq, yq):
    """Octave interp2(X, Y, F, xq, yq, 'linear') on a uniform grid."""
    hx = xv[1] - xv[0]
    hy = yv[1] - yv[0]
    ix = np.clip(np.floor((xq - xv[0]) / hx).astype(int), 0, len(xv) - 2)
    iy = np.clip(np.floor((yq - yv[0]) / hy).astype(int), 0, len(yv) - 2)
    tx = (xq - xv[ix]) / hx
    ty = (yq - yv[iy]) / hy
    f00 = F[iy, ix]
    f01 = F[iy, ix + 1]
    f10 = F[iy + 1, ix]
    f11 = F[iy + 1, ix + 1]
    return (1 - ty) * ((1 - tx) * f00 + tx * f01) + ty * ((1 - tx) * f10 + tx * f11)


def well_balance(nE: int = 50, L: float = 10.0, DX: float = 0.17, T: float = 1.0) -> DATA:
    hl = L / nE
    xv = _octave_range(0.0, hl, L)
    yv = _octave_range(0.0, hl, L)
    Xg, Yg = np.meshgrid(xv, yv)
    Zplot = 5.0 * np.exp(-2 / 5.0 * ((Xg - 5) ** 2 + (Yg - 5) ** 2))
    gx, gy = _gradient(Zplot, hl, hl)
    h = 10.0 - Zplot
    h[h < 0] = 0
    xs = _octave_range(0.0, DX, L)
    xp, yp = _meshgrid_colmajor(xs, xs)
    hp = _interp2_linear(xv, yv, h, xp, yp)
    n = xp.shape[0]
    rho = 1200.0
    Ap = DX * DX * np.ones(n)
    arrays = _particles(xp, yp, hp, Ap, rho)
    arrays.update({"Z": Zplot.reshape(-1, order="F"), "dZdx": gx.reshape(-1, order="F"),
                   "dZdy": gy.reshape(-1, order="F")})
    sc = _base_scalars(Nex=len(xv) - 1, Ney=len(yv) - 1, hx=hl, hy=hl, rho=rho,
                       T=T, xi=200.0, mu=2000.0, phi=20.0, tauy=30.0,
                       BINGHAM_ON=0.0, FRICTION_ON=0.0, CFL=0.1, BC_FLAG=0,
                       MERGE_SPLIT_ON=1, eq_level=10.0, DT_FIXED=0.0, NSTEPS=100,
                       ms_alpha=1.3, ms_beta=0.3)
    return DATA(arrays, sc)


# ---------------------------------------------------------------------------
# data/conservation_test/conservation_test.m (inclined plane + bump)
# ---------------------------------------------------------------------------
def conservation_bump(T: float = 20.0) -> DATA:
    nelex, neley, Lx, Ly = 75, 30, 150.0, 20.0
    hx, hy = Lx / nelex, Ly / neley
    x = _octave_linspace(0.0, Lx, nelex + 1)
    y = _octave_linspace(0.0, Ly, neley + 1)
    X, Y = np.meshgrid(x, y)
    Z = 60 - (1 / 3.0) * X + 15.0 * np.exp(-((X - 50) ** 2) / 7 - ((Y - 10) ** 2) / 7)
    gx, gy = _gradient(Z, hx, hy)
    DX = DY = 0.45
    xs = _octave_range(DX / 2, DX, 20 - DX / 2)
    ys = _octave_range(DY / 2, DY, 20 - DY / 2)
    xp, yp = _meshgrid_colmajor(xs, ys)
    hp = 60 - _interp2_linear(x, y, Z, xp, yp)
    keep = hp > 1.0
    xp, yp, hp = xp[keep], yp[keep], hp[keep]
    edge = (xp < hx) | (xp > Lx - hx) | (yp < hy) | (yp > Ly - hy)
    xp, yp, hp = xp[~edge], yp[~edge], hp[~edge]
    n = xp.shape[0]
    rho = 1200.0
    Msys = np.sum(hp * DX * DY * rho)
    Mp = Msys / n * np.ones(n)
    Vp = Mp / rho
    Ap = Vp / hp
    z = np.zeros(n)
    arrays = {"x": xp, "y": yp, "Mp": Mp, "Ap": Ap, "vpx": z.copy(), "vpy": z.copy(),
              "hp": hp, "mom_px": z.copy(), "mom_py": z.copy(), "Vp": Vp,
              "Z": Z.reshape(-1, order="F"), "dZdx": gx.reshape(-1, order="F"),
              "dZdy": gy.reshape(-1, order="F")}
    sc = _base_scalars(Nex=nelex, Ney=neley, hx=hx, hy=hy, rho=rho, T=T, xi=200.0,
                       mu=10.0, phi=12.0, tauy=30.0, BINGHAM_ON=1.0, FRICTION_ON=1.0,
                       CFL=0.2, BC_FLAG=1, MERGE_SPLIT_ON=1, eq_level=0.0)
    return DATA(arrays, sc)


# ---------------------------------------------------------------------------
# benchmark workloads
# ---------------------------------------------------------------------------
def dam_break_flat(nsteps: int = 500) -> DATA:
    """Flat dam break: 64x64 cells of 0.25 m, water column x in [0,4],
    y in [0,16] with 2x2 particles per cell (Np = 4096), hp = 1, rho = 1000,
    dt 1e-3 fixed.  Rheology constants as data/dambreak/dambreak.m:103-110
    (inactive: BINGHAM_ON = FRICTION_ON = 0)."""
    N, h = 64, 0.25
    offs = np.array([0.25, 0.75]) * h
    xs = (np.arange(16)[:, None] * h + offs[None, :]).reshape(-1)
    ys = (np.arange(64)[:, None] * h + offs[None, :]).reshape(-1)
    xp, yp = _meshgrid_colmajor(xs, ys)
    n = xp.shape[0]
    hp = np.ones(n)
    Ap = (h * h / 4) * np.ones(n)
    arrays = _particles(xp, yp, hp, Ap, 1000.0)
    nn = (N + 1) * (N + 1)
    arrays.update({"Z": np.zeros(nn), "dZdx": np.zeros(nn), "dZdy": np.zeros(nn)})
    sc = _base_scalars(Nex=N, Ney=N, hx=h, hy=h, rho=1000.0, T=8.0, xi=200.0, mu=50.0,
                       phi=37.0, tauy=2000.0, BINGHAM_ON=0.0, FRICTION_ON=0.0, CFL=0.2,
                       BC_FLAG=1, MERGE_SPLIT_ON=0, eq_level=0.0, DT_FIXED=1e-3,
                       NSTEPS=nsteps)
    return DATA(arrays, sc)


def _bumpy_slope(Nex, Ney, h, slope, nbumps, amp, sig, rng, slope_ref=None):
    """Z = slope*(x_ref - x) + sum of Gaussian bumps; analytic gradient."""
    Lx, Ly = Nex * h, Ney * h
    xr = Lx if slope_ref is None else slope_ref
    x = np.arange(Nex + 1) * h
    y = np.arange(Ney + 1) * h
    A = rng.uniform(amp[0], amp[1], nbumps)
    S = rng.uniform(sig[0], sig[1], nbumps)
    cx = rng.uniform(0, Lx, nbumps)
    cy = rng.uniform(0, Ly, nbumps)
    # node order r + c*(Ney+1): y fastest
    X = np.repeat(x, Ney + 1)
    Y = np.tile(y, Nex + 1)
    Z = slope * (xr - X)
    dZdx = np.full_like(X, -slope)
    dZdy = np.zeros_like(X)
    for k in range(nbumps):
        e = A[k] * np.exp(-((X - cx[k]) ** 2 + (Y - cy[k]) ** 2) / (2 * S[k] ** 2))
        Z += e
        dZdx += e * (-(X - cx[k]) / S[k] ** 2)
        dZdy += e * (-(Y - cy[k]) / S[k] ** 2)
    return Z, dZdx, dZdy


def _ellipse_release(Nex, Ney, h, ppc_side, cx, cy, a, b, hpeak):
    """Particles on a ppc_side x ppc_side lattice per cell inside an
    ellipse; hp = hpeak*(1 - r^2) in the normalised radius r."""
    c0 = max(int(math.floor((cx - a) / h)), 0)
    c1 = min(int(math.ceil((cx + a) / h)), Nex)
    r0 = max(int(math.floor((cy - b) / h)), 0)
    r1 = min(int(math.ceil((cy + b) / h)), Ney)
    offs = (np.arange(ppc_side) + 0.5) / ppc_side * h
    xs = (np.arange(c0, c1)[:, None] * h + offs[None, :]).reshape(-1)
    ys = (np.arange(r0, r1)[:, None] * h + offs[None, :]).reshape(-1)
    xp, yp = _meshgrid_colmajor(xs, ys)
    r2 = ((xp - cx) / a) ** 2 + ((yp - cy) / b) ** 2
    keep = r2 < 1.0
    xp, yp, r2 = xp[keep], yp[keep], r2[keep]
    hp = hpeak * (1.0 - r2)
    Ap = (h / ppc_side) ** 2 * np.ones(xp.shape[0])
    return xp, yp, hp, Ap


def mudflow(N: int = 2048, h: float = 0.5, seed: int = DEFAULT_SEED,
            merge_split: bool = False, nsteps: int = 2000) -> DATA:
    """Mudflow on a seeded bumpy slope: Z = 0.3*(1024 - x) + 32 Gaussian
    bumps (A ~ U[0,20] m, sigma ~ U[10,60] m, centres uniform), analytic
    dZdx/dZdy.  Release ellipse with semi-axes 200 m (x) x 100 m (y) centred
    at x = 512 m, 150 m below the top edge (y = Ly - 150), 4x4 particles per
    cell (~4.02M particles at N = 2048), hp = 5*(1 - r^2), rho = 1800.
    Bingham (mu 50, tauy 500) + Voellmy (phi 20, xi 500), BC on, CFL 0.4.
    Smaller N keeps the same physical shapes scaled by N/2048."""
    rng = np.random.default_rng(seed)
    s = N / 2048.0
    L = N * h
    Z, dZdx, dZdy = _bumpy_slope(N, N, h, 0.3, 32, (0.0, 20.0), (10.0 * s, 60.0 * s),
                                 rng, slope_ref=L)
    xp, yp, hp, Ap = _ellipse_release(N, N, h, 4, 0.5 * L, L - 150.0 * s, 200.0 * s,
                                      100.0 * s, 5.0)
    arrays = _particles(xp, yp, hp, Ap, 1800.0)
    arrays.update({"Z": Z, "dZdx": dZdx, "dZdy": dZdy})
    A0 = (h / 4) ** 2
    sc = _base_scalars(Nex=N, Ney=N, hx=h, hy=h, rho=1800.0, T=1e30, xi=500.0, mu=50.0,
                       phi=20.0, tauy=500.0, BINGHAM_ON=1.0, FRICTION_ON=1.0, CFL=0.4,
                       BC_FLAG=1, MERGE_SPLIT_ON=1 if merge_split else 0, eq_level=0.0,
                       DT_FIXED=0.0, NSTEPS=nsteps,
                       ms_alpha=math.sqrt(2.0 * A0) / h, ms_beta=math.sqrt(0.5 * A0) / h,
                       ms_min_level=-2, ms_max_level=2, ms_call_interval=10,
                       ms_pair_dist=0.25 if merge_split else 0.0)
    return DATA(arrays, sc)


def crowded_cells(seed: int = 5, nsteps: int = 200) -> DATA:
    """Cells crowded with hundreds to thousands of particles, as a fixed-dt
    ensemble member that has gone unstable piles its particles against a
    wall: a 48 x 48 grid of 0.5 m cells on a bumpy slope, an elliptic release
    at 4 x 4 particles per cell, and four cells holding 700, 1500 (the same
    cell column), 5000 and 20000 particles at uniform random positions.
    Bingham + Voellmy, adaptive CFL 0.4."""
    rng = np.random.default_rng(seed)
    N, h = 48, 0.5
    L = N * h
    Z, dZdx, dZdy = _bumpy_slope(N, N, h, 0.3, 8, (0.0, 2.0), (1.0, 4.0), rng, slope_ref=L)
    xp, yp, hp, Ap = _ellipse_release(N, N, h, 4, 0.5 * L, 0.5 * L, 6.0, 4.0, 2.0)
    xs, ys, hs, As = [xp], [yp], [hp], [Ap]
    for col, row, m in ((20, 10, 700), (20, 14, 1500), (30, 24, 5000), (40, 40, 20000)):
        xs.append((col + rng.uniform(0.02, 0.98, m)) * h)
        ys.append((row + rng.uniform(0.02, 0.98, m)) * h)
        hs.append(np.full(m, 0.5))
        As.append(np.full(m, h * h / m))
    arrays = _particles(np.concatenate(xs), np.concatenate(ys), np.concatenate(hs),
                        np.concatenate(As), 1800.0)
    arrays.update({"Z": Z, "dZdx": dZdx, "dZdy": dZdy})
    sc = _base_scalars(Nex=N, Ney=N, hx=h, hy=h, rho=1800.0, T=1e30, xi=500.0, mu=50.0,
                       phi=20.0, tauy=500.0, BINGHAM_ON=1.0, FRICTION_ON=1.0, CFL=0.4,
                       BC_FLAG=1, MERGE_SPLIT_ON=0, eq_level=0.0, DT_FIXED=0.0,
                       NSTEPS=nsteps)
    return DATA(arrays, sc)


def ensemble_member(seed: int, side_range=(64, 512), h: float = 1.0,
                    dt: float = 0.02, nsteps: int = 1000) -> DATA:
    """One scenario of the batched ensemble: square grid (side log-uniform),
    slope U[0.2,0.5] + 8 bumps (A ~ U[0,15], sigma ~ U[5,40]), release
    ellipse covering 2-10 % of the domain at 4 particles per cell, parabolic
    hp with peak U[2,8] m; rho, mu, tauy, phi, xi uniform in the configured
    ranges; fixed dt."""
    rng = np.random.default_rng(seed)
    side = int(round(math.exp(rng.uniform(math.log(side_range[0]), math.log(side_range[1])))))
    slope = rng.uniform(0.2, 0.5)
    L = side * h
    Z, dZdx, dZdy = _bumpy_slope(side, side, h, slope, 8, (0.0, 15.0), (5.0, 40.0), rng,
                                 slope_ref=L)
    frac = rng.uniform(0.02, 0.10)
    area = frac * L * L
    ratio = rng.uniform(1.0, 2.0)
    b = math.sqrt(area / (math.pi * ratio))
    a = ratio * b
    a = min(a, 0.45 * L)
    b = min(b, 0.45 * L)
    cx = rng.uniform(a + h, L - a - h) if L - 2 * a - 2 * h > 0 else 0.5 * L
    cy = rng.uniform(b + h, L - b - h) if L - 2 * b - 2 * h > 0 else 0.5 * L
    hpeak = rng.uniform(2.0, 8.0)
    xp, yp, hp, Ap = _ellipse_release(side, side, h, 2, cx, cy, a, b, hpeak)
    rho = rng.uniform(1500.0, 2200.0)
    arrays = _particles(xp, yp, hp, Ap, rho)
    arrays.update({"Z": Z, "dZdx": dZdx, "dZdy": dZdy})
    sc = _base_scalars(Nex=side, Ney=side, hx=h, hy=h, rho=rho, T=nsteps * dt,
                       xi=rng.uniform(200.0, 2000.0), mu=rng.uniform(10.0, 200.0),
                       phi=rng.uniform(15.0, 35.0), tauy=rng.uniform(100.0, 2000.0),
                       BINGHAM_ON=1.0, FRICTION_ON=1.0, CFL=0.4, BC_FLAG=1,
                       MERGE_SPLIT_ON=0, eq_level=0.0, DT_FIXED=dt, NSTEPS=nsteps)
    return DATA(arrays, sc)


def serving_request(seed: int, t_end: float = 60.0) -> DATA:
    """A serving request: as an ensemble member with side log-uniform in
    [64, 1024] cells, run with adaptive CFL 0.4 to t_end."""
    d = ensemble_member(seed, side_range=(64, 1024))
    d.scalars.update({"DT_FIXED": 0.0, "T": float(t_end), "CFL": 0.4, "NSTEPS": 0})
    return d
