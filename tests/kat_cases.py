"""The known-answer cases: each builds a world (kat_worlds), runs it through a stepping
callable (the oracle on the CPU, the CUDA step on the GPU) and checks the result against an
answer computed here without the oracle.

- `ogden_*`: four stretched latex triangles off the water, no gravity. One step of 40 ns moves
  them by about 1e-6 of their size, so each vertex's velocity after the step is dt / m times
  the elastic force, which is compared with the force from the closed form of the reference's
  `Latex::stress` (src/balloon.rs:31-71, f64; membrane.wgsl:50-149 is the kernel under test).
- `sod_*`: a shock tube in the air (air.wgsl:150-269, HLL fluxes) against the exact solution of
  the Riemann problem.
- `hydro_*`: a wide water layer on the ground with gravity and a sound speed so high that the
  water is incompressible: the solved pressure is rho g (depth) cell by cell
  (fluid.wgsl:445-598).
- `pcg_*`: a water box carrying a manufactured pressure field; the pressure system the step
  assembles is rebuilt here from the step's own transfer sums and cell types and solved with a
  sparse direct solver in f64, and the step's PCG solution is compared with it
  (fluid.wgsl:381-578).
- `advect_*`: a block of water moving at a uniform velocity with no gravity translates
  unchanged (fluid.wgsl:198-303 and 767-901).
"""
from __future__ import annotations

import math

import numpy as np

from kat_worlds import (A_PC, A_WC, F_P, F_TYPE, F_U, FP_M, FP_P, FP_W, GAS, GAMMA, P_ATM, RHO_ATM, SOLID, WATER,
                        all_blocks, assemble, cell_coords, header, lattice, no_membrane, particles)

# ---------------------------------------------------------------------------------------------
# Ogden latex triangles against Latex::stress
# ---------------------------------------------------------------------------------------------
OGDEN_ALPHA = (1.3, 5.0, -2.0)
OGDEN_DT = 4e-8
EDGE = 1e-3
RHO_RUBBER = 950.0

# In-plane deformation of each triangle (2x2, applied to the rest triangle's plane coordinates):
# taut both ways, pulled one way and wrinkled across, slack, and sheared (principal directions
# off the rest axes).
OGDEN_CASES = {
    "biaxial": [[2.5, 0.0], [0.0, 1.8]],
    "wrinkled": [[3.0, 0.0], [0.0, 0.5]],
    "slack": [[0.9, 0.0], [0.0, 0.8]],
    "sheared": [[2.0, 0.7], [0.3, 1.6]],
}


def _rotation(a: float, b: float, c: float) -> np.ndarray:
    ca, sa, cb, sb, cc, sc = math.cos(a), math.sin(a), math.cos(b), math.sin(b), math.cos(c), math.sin(c)
    rx = np.array([[1, 0, 0], [0, ca, -sa], [0, sa, ca]])
    ry = np.array([[cb, 0, sb], [0, 1, 0], [-sb, 0, cb]])
    rz = np.array([[cc, -sc, 0], [sc, cc, 0], [0, 0, 1]])
    return rz @ ry @ rx


def ogden_world():
    h_cell, blocks, origin = 2e-3, (16, 16, 16), (0.0, 0.5, 0.0)
    rest = np.array([[0.0, 0.0], [EDGE, 0.0], [0.5 * EDGE, 0.5 * math.sqrt(3.0) * EDGE]])
    dm = np.stack([rest[1] - rest[0], rest[2] - rest[0]], 1)  # columns: the rest edges
    dm_inv = np.linalg.inv(dm)
    area = 0.5 * abs(np.linalg.det(dm))
    ref = header(h_cell, origin, blocks, n_particles=1, n_verts=1, n_tris=0, n_vtri=0)
    thick = float(np.float32(ref.params.rubber[3]))
    mass = np.float32(RHO_RUBBER * thick * area / 3.0)
    n = len(OGDEN_CASES)
    xs, tris, cases = [], [], []
    for k, (name, g) in enumerate(OGDEN_CASES.items()):
        rot = _rotation(0.3 + 0.4 * k, -0.2 + 0.3 * k, 0.5 * k)
        centre = np.array([origin[0] + 0.02 + 0.025 * k, origin[1] + 0.064, origin[2] + 0.064])
        x = np.array([centre + rot @ np.array([*(np.array(g) @ r), 0.0]) for r in rest])
        xs.append(x)
        tris.append([3 * k, 3 * k + 1, 3 * k + 2])
        cases.append(name)
    x = np.concatenate(xs).astype(np.float32)
    h = header(h_cell, origin, blocks, n_particles=1, n_verts=3 * n, n_tris=n, n_vtri=3 * n, dt_max=OGDEN_DT)
    tri = np.zeros((n, 8), np.uint32)
    tri[:, :3] = np.array(tris, np.uint32)
    tri[:, 3] = np.float32(area).view(np.uint32)
    tri[:, 4:8] = np.array(dm_inv.reshape(-1), np.float32).view(np.uint32)  # row-major
    secs = {
        "PARTICLES": particles(np.array([[0.01, 0.51, 0.01]], np.float32), alive=0.0),
        "MEM_X": np.concatenate([x, np.zeros((3 * n, 1), np.float32)], 1),
        "MEM_MASS": np.full(3 * n, mass, np.float32),
        "MEM_PUSH": np.tile(np.array([0.0, area / 3.0], np.float32), (3 * n, 1)),
        "TRIS": tri, "ALIVE": np.ones(n, np.uint32),
        "VTRI_OFF": np.arange(3 * n + 1, dtype=np.uint32), "VTRI": np.repeat(np.arange(n, dtype=np.uint32), 3),
    }
    return assemble(h, secs), dict(cases=cases, mass=float(mass), dm_inv=dm_inv, area=area, thick=thick, x0=x.astype(np.float64))


def latex_stress(mu, l1: float, l2: float) -> tuple[float, float]:
    """`Latex::stress` of src/balloon.rs:51-63 in f64: the principal Cauchy stresses of an
    incompressible Ogden sheet in plane stress, wrinkled (pulled one way only) or slack where
    it would be squeezed in its plane."""
    def sigma(a, b):
        return sum(m * (a ** al - b ** al) for m, al in zip(mu, OGDEN_ALPHA))
    major, minor = max(l1, l2), min(l1, l2)
    if major <= 1.0:
        return 0.0, 0.0
    natural = major ** -0.5
    if minor < natural:
        s = sigma(major, natural)
        return (s, 0.0) if l1 >= l2 else (0.0, s)
    l3 = 1.0 / (l1 * l2)
    return sigma(l1, l3), sigma(l2, l3)


def ogden_expected_forces(x: np.ndarray, mu, info) -> np.ndarray:
    """Vertex forces of the triangle at positions x (3 x 3, f64) under the uniform stress of its
    deformation: f = -V0 P grad N with P = F S, S = sum sigma_i / l_i^2 N_i N_i^T."""
    g = info["dm_inv"]
    F = np.stack([x[1] - x[0], x[2] - x[0]], 1) @ g  # 3 x 2
    lam2, N = np.linalg.eigh(F.T @ F)
    lam = np.sqrt(np.maximum(lam2, 0.0))
    s1, s2 = latex_stress(mu, lam[1], lam[0])  # eigh sorts ascending
    S = s1 / lam[1] ** 2 * np.outer(N[:, 1], N[:, 1]) + s2 / lam[0] ** 2 * np.outer(N[:, 0], N[:, 0])
    P = F @ S
    v0 = info["area"] * info["thick"]
    f1 = -v0 * P @ g[0]
    f2 = -v0 * P @ g[1]
    return np.stack([-(f1 + f2), f1, f2])


def check_ogden(w0, info, w1) -> dict:
    """Forces measured from the step's velocities against the closed form; returns the worst
    relative error per case."""
    mu = [float(v) for v in w0.h.params.rubber[:3]]
    dt = w1.state["dt_ns"] * 1e-9
    assert w1.state["dt_ns"] == round(OGDEN_DT * 1e9)
    v = w1.sec("MEM_V")[:, :3].astype(np.float64)
    out = {}
    scale = 0.0
    for k, name in enumerate(info["cases"]):
        want = ogden_expected_forces(info["x0"][3 * k: 3 * k + 3], mu, info)
        got = v[3 * k: 3 * k + 3] * info["mass"] / dt
        scale = max(scale, float(np.abs(want).max()))
        out[name] = (got, want)
    errs = {}
    for name, (got, want) in out.items():
        # Relative to the largest force of the scene (the slack triangle's is zero).
        errs[name] = float(np.abs(got - want).max() / scale)
    return errs


# ---------------------------------------------------------------------------------------------
# Sod shock tube against the exact Riemann solution
# ---------------------------------------------------------------------------------------------
SOD_H = 0.01
SOD_BLOCKS = (24, 32, 32)  # 96 cells along the tube, 128 x 128 across
SOD_X0 = 48  # the membrane between the two states, in cells
SOD_LEFT = (8.0 * RHO_ATM, 10.0 * P_ATM)
# The right state is 100 Pa above the ambient air, so that every block of the tube counts as
# active air (air.wgsl:264: more than 10 Pa from ambient) and stays allocated: the step keeps
# only the blocks whose air is doing something, and the air past them is ambient.
SOD_RIGHT = (RHO_ATM, P_ATM + 100.0)
SOD_DT = 2e-5
SOD_STEPS = 10


def sod_world():
    blocks = SOD_BLOCKS
    origin = (0.0, 1.0, 0.0)
    bl = all_blocks(blocks)
    nc = bl.size * 64
    c = cell_coords(bl, blocks)
    left = c[:, 0] < SOD_X0
    rho = np.where(left, SOD_LEFT[0], SOD_RIGHT[0]).astype(np.float32)
    p = np.where(left, SOD_LEFT[1], SOD_RIGHT[1]).astype(np.float32)
    air = np.zeros((5, nc), np.float32)
    air[0] = rho
    air[4] = p / np.float32(GAMMA - 1.0)
    h = header(SOD_H, origin, blocks, n_particles=1, n_verts=1, n_tris=0, n_vtri=0, n_blocks_prev=bl.size,
               dt_max=SOD_DT, air_substeps=4)
    centre = (origin[0] + 0.5 * SOD_H, origin[1] + 0.5 * SOD_H, origin[2] + 0.5 * SOD_H)
    secs = {"PARTICLES": particles(np.array([centre], np.float32), alive=0.0), **no_membrane(centre),
            "BLOCKS_PREV": bl, "BLOCK_ACTIVE": np.ones(bl.size, np.uint32), "AIR": air}
    return assemble(h, secs), dict(blocks=blocks)


def riemann_exact(left, right, xi: np.ndarray, gamma: float = GAMMA) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Exact solution of the Riemann problem of the Euler equations for an ideal gas, at the
    similarity coordinates xi = (x - x0) / t (Toro, Riemann Solvers and Numerical Methods for
    Fluid Dynamics, ch. 4: the star pressure by Newton's method on the pressure function, then
    the wave pattern sampled). States are (rho, p) at rest. Returns rho, u, p."""
    rl, pl = left
    rr, pr = right
    ul = ur = 0.0
    cl, cr = math.sqrt(gamma * pl / rl), math.sqrt(gamma * pr / rr)
    g1 = (gamma - 1.0) / (2.0 * gamma)

    def f(p, rk, pk, ck):
        if p > pk:  # shock
            a, b = 2.0 / ((gamma + 1.0) * rk), (gamma - 1.0) / (gamma + 1.0) * pk
            q = math.sqrt(a / (p + b))
            return (p - pk) * q, q * (1.0 - 0.5 * (p - pk) / (p + b))
        pr_ = (p / pk) ** g1  # rarefaction
        return 2.0 * ck / (gamma - 1.0) * (pr_ - 1.0), 1.0 / (rk * ck) * (p / pk) ** (-(gamma + 1.0) / (2.0 * gamma))

    p = 0.5 * (pl + pr)
    for _ in range(100):
        fl, dl = f(p, rl, pl, cl)
        fr, dr = f(p, rr, pr, cr)
        dp = (fl + fr + ur - ul) / (dl + dr)
        p = max(p - dp, 1e-8)
        if abs(dp) < 1e-14 * p:
            break
    fl, _ = f(p, rl, pl, cl)
    fr, _ = f(p, rr, pr, cr)
    u = 0.5 * (ul + ur) + 0.5 * (fr - fl)
    rho, uu, pp = np.empty_like(xi), np.empty_like(xi), np.empty_like(xi)
    gm = (gamma - 1.0) / (gamma + 1.0)
    # Left: a rarefaction (p* < pl for these states), right: a shock.
    assert p < pl and p > pr
    rho_l_star = rl * (p / pl) ** (1.0 / gamma)
    c_l_star = cl * (p / pl) ** g1
    head, tail = ul - cl, u - c_l_star
    rho_r_star = rr * ((p / pr + gm) / (gm * p / pr + 1.0))
    s_shock = ur + cr * math.sqrt((gamma + 1.0) / (2.0 * gamma) * p / pr + g1)
    for i, s in enumerate(xi):
        if s < head:
            rho[i], uu[i], pp[i] = rl, ul, pl
        elif s < tail:
            uf = 2.0 / (gamma + 1.0) * (cl + 0.5 * (gamma - 1.0) * ul + s)
            cf = 2.0 / (gamma + 1.0) * (cl + 0.5 * (gamma - 1.0) * (ul - s))
            rho[i], uu[i], pp[i] = rl * (cf / cl) ** (2.0 / (gamma - 1.0)), uf, pl * (cf / cl) ** (1.0 / g1)
        elif s < u:
            rho[i], uu[i], pp[i] = rho_l_star, u, p
        elif s < s_shock:
            rho[i], uu[i], pp[i] = rho_r_star, u, p
        else:
            rho[i], uu[i], pp[i] = rr, ur, pr
    return rho, uu, pp, dict(p_star=p, u_star=u, shock=s_shock, head=head, tail=tail, contact=u)


def sod_profiles(w1, info):
    """Density, velocity and pressure along the tube's centre line, and how far the cells of the
    core (the 17 x 17 lines around it) differ from it."""
    blocks = info["blocks"]
    bl = w1.sec("BLOCKS_PREV")
    air = w1.sec("AIR").reshape(5, -1).astype(np.float64)
    c = cell_coords(bl, blocks)
    ny, nz = 4 * blocks[1], 4 * blocks[2]
    mid = ny // 2
    nx = 4 * blocks[0]
    # Blocks the step no longer keeps hold the still air at atmospheric pressure, as the step
    # takes them to (the right state is exactly that air).
    grid = np.empty((5, nx, ny, nz))
    grid[0], grid[1:4], grid[4] = RHO_ATM, 0.0, P_ATM / (GAMMA - 1.0)
    grid[:, c[:, 0], c[:, 1], c[:, 2]] = air
    rho = grid[0]
    u = grid[1] / rho
    e = grid[4]
    p = (GAMMA - 1.0) * (e - 0.5 * (grid[1] ** 2 + grid[2] ** 2 + grid[3] ** 2) / rho)
    core = slice(mid - 8, mid + 9)
    spread = float(np.max(np.abs(rho[:, core, core] - rho[:, mid:mid + 1, mid:mid + 1])) / SOD_LEFT[0])
    return rho[:, mid, mid], u[:, mid, mid], p[:, mid, mid], spread


def check_sod(w1, info) -> dict:
    t = w1.state["t_ns"] * 1e-9
    rho, u, p, spread = sod_profiles(w1, info)
    x = (np.arange(rho.size) + 0.5 - SOD_X0) * SOD_H  # cell centres relative to the initial jump
    er, eu, ep, waves = riemann_exact(SOD_LEFT, SOD_RIGHT, x / t)
    # Where the waves are, and a margin of 3 cells beyond the outermost.
    lo = int(math.floor(SOD_X0 + waves["head"] * t / SOD_H)) - 3
    hi = int(math.ceil(SOD_X0 + waves["shock"] * t / SOD_H)) + 3
    sl = slice(max(lo, 0), min(hi, rho.size))
    l1 = lambda a, b, s: float(np.abs(a[sl] - b[sl]).mean() / s)
    # The star region away from its two ends (the rarefaction's tail and the shock), where the
    # first-order scheme's smearing has died out: pressure and velocity there are p*, u*.
    a = int(math.ceil(SOD_X0 + waves["tail"] * t / SOD_H)) + 2
    b = int(math.floor(SOD_X0 + waves["shock"] * t / SOD_H)) - 3
    plateau = slice(a, b)
    # Where the numerical shock is: the first cell from the right whose pressure is above the
    # mid value between the star and the right pressure.
    pmid = 0.5 * (waves["p_star"] + SOD_RIGHT[1])
    above = np.nonzero(p > pmid)[0]
    shock_cell = float(above.max()) + 0.5 - SOD_X0 if above.size else float("nan")
    return dict(t=t, l1_rho=l1(rho, er, SOD_LEFT[0]), l1_u=l1(u, eu, waves["u_star"]), l1_p=l1(p, ep, SOD_LEFT[1]),
                plateau_p=float(np.abs(p[plateau] / waves["p_star"] - 1.0).max()),
                plateau_u=float(np.abs(u[plateau] / waves["u_star"] - 1.0).max()),
                plateau_cells=b - a, shock_err_cells=abs(shock_cell - waves["shock"] * t / SOD_H),
                core_spread=spread, shock_cells=waves["shock"] * t / SOD_H)


# ---------------------------------------------------------------------------------------------
# The pressure system: assembled again from the step's own inputs and solved in f64
# ---------------------------------------------------------------------------------------------
def _index_of(coords: np.ndarray, dims) -> np.ndarray:
    """Dense map from domain cell coordinates to storage index (-1 where no cell is allocated)."""
    m = np.full(tuple(dims), -1, np.int64)
    m[coords[:, 0], coords[:, 1], coords[:, 2]] = np.arange(len(coords))
    return m


def pressure_system(grid: dict, w0, dt: float):
    """The scaled pressure equation of the step (fluid.wgsl:445-491), rebuilt from the step's
    transfer sums (acc), its cell types and the gas pressures, in f64: A p = b over the water
    cells, with the cell velocities u* = momentum / weight + g dt (grid_prep, fluid.wgsl:319-356),
    the divergence of the faces bounded at the ground, the carried pressures as p_old, and the
    gas (and outside) neighbours as known pressures. Returns (A, b, water cell indices, the
    step's solved pressure there)."""
    import scipy.sparse as sp
    P = w0.h.params
    blocks = tuple(int(v) for v in P.bdims[:3])
    dims = tuple(4 * b for b in blocks)
    bl = grid["block_list"]
    n = bl.size * 64
    acc = grid["acc"].reshape(19, n)
    cf = grid["cf"].reshape(11, n)
    ty = cf[F_TYPE]
    coords = cell_coords(bl, blocks)
    idx = _index_of(coords, dims)
    f32 = np.float32
    h = f32(P.origin[3])
    rho = f32(P.fluid[0])
    g = [f32(P.gravity[k]) for k in range(3)]
    dt32 = f32(dt)
    # u* of each cell's three low faces.
    u = np.zeros((3, n), np.float32)
    for d in range(3):
        wt = acc[2 * d + 1].astype(np.float32) / f32(FP_W)
        mom = acc[2 * d].astype(np.float32) / f32(FP_M)
        ok = wt > f32(1e-6)
        u[d, ok] = mom[ok] / wt[ok] + dt32 * g[d]
    # p_old: the carried pressure of the water cells (grid_prep).
    wc = acc[A_WC].astype(np.float32) / f32(FP_W)
    p_old = np.zeros(n, np.float32)
    okp = (ty == f32(WATER)) & (wc > f32(1e-6))
    p_old[okp] = acc[A_PC][okp].astype(np.float32) / f32(FP_P) / wc[okp] * f32(1e6)

    def nb(cells, d, s):
        q = coords[cells].copy()
        q[:, d] += s
        inside = np.all((q >= 0) & (q < np.array(dims)), 1)
        out = np.full(len(cells), -1, np.int64)
        out[inside] = idx[q[inside, 0], q[inside, 1], q[inside, 2]]
        return out

    def type_of(j):
        return np.where(j < 0, GAS, ty[np.maximum(j, 0)]).astype(np.float64)

    def face_u(hi, lo, d):
        """u of the face between `lo` and `hi` along d, bounded at solid cells (fluid.wgsl:358-366)."""
        v = np.where(hi < 0, 0.0, u[d, np.maximum(hi, 0)].astype(np.float64))
        th, tl = type_of(hi), type_of(lo)
        v = np.where((th == SOLID) & (tl == SOLID), 0.0, v)
        v = np.where((tl == SOLID) & (th != SOLID), np.maximum(v, 0.0), v)
        v = np.where((th == SOLID) & (tl != SOLID), np.minimum(v, 0.0), v)
        return np.where(hi < 0, 0.0, v)

    water = np.nonzero(ty == f32(WATER))[0]
    pos = np.full(n, -1, np.int64)
    pos[water] = np.arange(water.size)
    cs = f32(P.gravity[3]) * dt32
    kc = float(h * h / (cs * cs))
    diag = np.full(water.size, kc)
    b = kc * p_old[water].astype(np.float64)
    div = np.zeros(water.size)
    rows, cols = [], []
    for d in range(3):
        up, dn = nb(water, d, +1), nb(water, d, -1)
        div += face_u(up, water, d) - face_u(water, dn, d)
        for j in (up, dn):
            t = type_of(j)
            open_ = t != SOLID
            diag += open_
            wn = open_ & (t == WATER)
            rows.append(np.nonzero(wn)[0])
            cols.append(pos[j[wn]])
            known = open_ & (t != WATER)
            pk = np.where(j < 0, 0.0, cf[F_P, np.maximum(j, 0)].astype(np.float64))
            b += np.where(known, pk, 0.0)
    b -= float(rho) * float(h) / float(dt32) * div
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    A = sp.csr_matrix((np.concatenate([diag, -np.ones(r.size)]), (np.concatenate([np.arange(water.size), r]),
                                                                    np.concatenate([np.arange(water.size), c]))),
                      shape=(water.size, water.size))
    return A, b, water, cf[F_P, water].astype(np.float64), coords


def check_pressure_system(grid, w0, dt) -> dict:
    import scipy.sparse.linalg as spla
    A, b, water, p_step, _ = pressure_system(grid, w0, dt)
    p_ref = spla.spsolve(A.tocsc(), b)
    return dict(n_water=int(water.size), rel_err=float(np.linalg.norm(p_step - p_ref) / np.linalg.norm(p_ref)),
                rel_residual=float(np.linalg.norm(A @ p_step - b) / np.linalg.norm(b)), p_ref=p_ref, p_step=p_step)


PCG_BOX = (24, 24, 24)


def pcg_world(solve_tol: float = 1e-6):
    """A water box at rest, no gravity, carrying a smooth manufactured pressure field."""
    h_cell, blocks, origin = 2e-3, (10, 10, 10), (0.0, 0.5, 0.0)
    lo = (8, 8, 8)
    hi = tuple(a + b for a, b in zip(lo, PCG_BOX))
    pos = lattice(lo, hi, h_cell, origin)
    rel = (pos.astype(np.float64) - np.array(origin)) / h_cell
    pres = (4000.0 * np.sin(0.31 * rel[:, 0]) * np.cos(0.23 * rel[:, 1] + 0.4) + 2500.0 * np.sin(0.17 * rel[:, 2] + 1.1)
            + 1500.0).astype(np.float32)
    h = header(h_cell, origin, blocks, n_particles=len(pos), n_verts=1, n_tris=0, n_vtri=0, iters=4096,
               solve_tol=solve_tol)
    secs = {"PARTICLES": particles(pos, pressure=pres), **no_membrane(origin)}
    return assemble(h, secs), {}


HYDRO_W, HYDRO_D = 96, 4  # cells across and deep


def hydro_world(solve_tol: float = 1e-6):
    """A wide water layer HYDRO_D cells deep on the ground, at rest under gravity, with a sound
    speed of 1e7 m/s: the compressible term of the pressure equation vanishes and the pressure
    is hydrostatic. The ground is the block of cells below y = 0 (solid, fluid.wgsl:305-307)."""
    h_cell = 2e-3
    blocks = (HYDRO_W // 4, 4, HYDRO_W // 4)
    origin = (0.0, -4 * h_cell, 0.0)
    pos = lattice((0, 4, 0), (HYDRO_W, 4 + HYDRO_D, HYDRO_W), h_cell, origin)
    h = header(h_cell, origin, blocks, n_particles=len(pos), n_verts=1, n_tris=0, n_vtri=0, iters=4096,
               gravity=(0.0, -9.81, 0.0), sound_speed=1e7, solve_tol=solve_tol)
    secs = {"PARTICLES": particles(pos), **no_membrane((0.0, 0.5, 0.0))}
    return assemble(h, secs), {}


def check_hydro(grid, w0) -> dict:
    """The step's pressure in the water cells of the middle of the layer (16 x 16 columns, 40
    cells from its edges) against p_gas + rho |g| h (cells from the top + 1), the discrete
    hydrostatic solution with the gas above as the known pressure."""
    P = w0.h.params
    blocks = tuple(int(v) for v in P.bdims[:3])
    bl = grid["block_list"]
    cf = grid["cf"].reshape(11, -1)
    c = cell_coords(bl, blocks)
    idx = _index_of(c, tuple(4 * b for b in blocks))
    rho, g, h = float(P.fluid[0]), -float(P.gravity[1]), float(P.origin[3])
    mid = HYDRO_W // 2
    worst, worst_v = 0.0, 0.0
    for x in range(mid - 8, mid + 8):
        for z in range(mid - 8, mid + 8):
            top = 4 + HYDRO_D  # the gas cell above the layer
            p_gas = float(cf[F_P, idx[x, top, z]])
            assert cf[F_TYPE, idx[x, top, z]] == GAS
            for y in range(4, top):
                k = idx[x, y, z]
                assert cf[F_TYPE, k] == WATER
                want = p_gas + rho * g * h * (top - y)
                worst = max(worst, abs(float(cf[F_P, k]) - want) / (rho * g * h * HYDRO_D))
                worst_v = max(worst_v, abs(float(cf[F_U + 1, k])))
    return dict(rel_err=worst, max_v=worst_v)


ADV_V = (0.3, -0.2, 0.1)
ADV_STEPS = 20


def advect_world():
    """A 16^3-cell block of water moving at ADV_V, no gravity."""
    h_cell, blocks, origin = 2e-3, (10, 10, 10), (0.0, 0.5, 0.0)
    pos = lattice((12, 12, 12), (28, 28, 28), h_cell, origin)
    vel = np.tile(np.array(ADV_V, np.float32), (len(pos), 1))
    h = header(h_cell, origin, blocks, n_particles=len(pos), n_verts=1, n_tris=0, n_vtri=0, iters=4096)
    secs = {"PARTICLES": particles(pos, vel=vel), **no_membrane(origin)}
    return assemble(h, secs), dict(x0=pos.astype(np.float64))


def check_advect(w1, info, grid=None) -> dict:
    """Velocities against ADV_V (relative to |ADV_V|), positions against x0 + dt v in f32 after
    the first step, and the grid's face velocities where the particles' weight is at least 0.01."""
    p = w1.particles.astype(np.float64)
    V = np.array(ADV_V)
    vmag = float(np.linalg.norm(V))
    out = dict(t=w1.state["t_ns"] * 1e-9, dv=float(np.abs(p[:, 4:7] - V).max() / vmag),
               alive=int((p[:, 7] > 0.5).sum()), n=len(p),
               # the affine terms stay zero (c0..c2 xyz)
               affine=float(np.abs(p[:, [8, 9, 10, 12, 13, 14, 16, 17, 18]]).max()))
    if w1.state["step"] == 1:
        dt = np.float32(w1.state["dt_ns"] * 1e-9)
        want = info["x0"].astype(np.float32) + p[:, 4:7].astype(np.float32) * dt
        out["dx_f32"] = float(np.abs(p[:, :3] - want.astype(np.float64)).max())
    if grid is not None:
        n = grid["block_list"].size * 64
        acc, cf = grid["acc"].reshape(19, n), grid["cf"].reshape(11, n)
        out["grid_du"] = max(float(np.abs(cf[F_U + d][acc[2 * d + 1] > 0.01 * FP_W] - V[d]).max() / vmag) for d in range(3))
    return out
