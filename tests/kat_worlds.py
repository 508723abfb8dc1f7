"""Known-answer worlds: scenes assembled section by section, for tests whose expected result
comes from outside the oracle (an exact Riemann solution, hydrostatics, an independent sparse
solve of the pressure system, the Ogden closed form of src/balloon.rs, uniform translation).

A world blob is the header followed by the sections at 256-byte aligned offsets, in section
order (the layout `ntr_world_build` writes; include/natray.h lists the sections). These scenes
have no bullets, keep one dead particle where they need no water and one massless vertex where
they need no membrane (the step's launches are sized from both counts), and set the substep
counts in the header so that no measuring substep runs at creation: the CUDA step and the oracle
start from exactly these bytes.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from natray_b200 import Params, World, build_world
from natray_b200._abi import LAYER_MODES, MAX_SHOTS, SECTIONS, WORLD_MAGIC, WORLD_VERSION, WorldHeader

FLT_MAX = float(np.finfo(np.float32).max)
GAS, WATER, SOLID = 0.0, 1.0, 2.0  # cell types (shaders/sim_defs.wgsl:152-157)
F_U, F_P, F_TYPE = 0, 3, 10  # cell fields used here (velocity x,y,z; pressure; type)
A_WC, A_PC = 6, 7  # transfer sums: cell weight and weighted pressure
FP_M, FP_W, FP_P = 65536.0, 16777216.0, 65536.0
P_ATM, RHO_ATM, GAMMA = 101325.0, 1.204, 1.4

_REF = None


def _reference_params():
    """Material constants of the default scene (Ogden moduli of `Latex::new`, friction, break
    stretch, wet map size), taken from a built world so the known-answer scenes use the same."""
    global _REF
    if _REF is None:
        _REF = build_world(Params(resolution=16, mesh_level=1)).h.params
    return _REF


def _shape(h: WorldHeader, name: str) -> tuple[int, int]:
    cells_prev = h.n_blocks_prev * 64
    return {
        "PARTICLES": (80, h.n_particles), "MEM_X": (16, h.n_verts), "MEM_V": (16, h.n_verts), "MEM_MASS": (4, h.n_verts),
        "MEM_WATER": (16, h.n_verts), "MEM_LAYER": (16 * LAYER_MODES, h.n_verts), "MEM_PUSH": (8, h.n_verts),
        "TRIS": (32, h.n_tris), "ALIVE": (4, h.n_tris), "VTRI_OFF": (4, h.n_verts + 1), "VTRI": (4, h.n_vtri),
        "BULLETS": (112, MAX_SHOTS), "PATCHES": (32, MAX_SHOTS * 576), "OUTLINES": (8, MAX_SHOTS * 33),
        "SECTIONS": (48, MAX_SHOTS * 32), "BULLET_HIT": (4, MAX_SHOTS * 13), "POSE_LOG": (48, MAX_SHOTS * 256),
        "BLOCKS_PREV": (4, h.n_blocks_prev), "BLOCK_ACTIVE": (4, h.n_blocks_prev), "AIR": (4, 5 * cells_prev),
        "SPRAY": (48, h.n_spray), "LANDED": (16, h.n_spray), "TOUCH": (4, h.wet_res * h.wet_res),
    }[name]


def assemble(h: WorldHeader, secs: dict[str, np.ndarray]) -> World:
    """The blob of header `h` with the given sections (the rest zero)."""
    off = (C.sizeof(WorldHeader) + 255) & ~255
    data = []
    for i, name in enumerate(SECTIONS):
        elem, count = _shape(h, name)
        want = elem * count
        a = secs.get(name)
        raw = np.zeros(want, np.uint8) if a is None else np.ascontiguousarray(a).view(np.uint8).reshape(-1)
        assert raw.size == want, f"section {name}: {raw.size} bytes, expected {want}"
        h.offset[i], h.bytes[i] = off, want
        data.append((off, raw))
        off += (want + 255) & ~255
    blob = bytearray(off)
    blob[: C.sizeof(WorldHeader)] = bytes(h)
    for o, raw in data:
        blob[o: o + raw.size] = raw.tobytes()
    return World(blob, copy=False)


def header(h_cell: float, origin, blocks, *, n_particles: int, n_verts: int, n_tris: int, n_vtri: int,
           n_blocks_prev: int = 0, block_cap: int = 65535, dt_max: float = 2e-6, gravity=(0.0, 0.0, 0.0),
           sound_speed: float = 1480.0, substeps: int = 2, air_substeps: int = 2, iters: int = 64,
           solve_tol: float = 1e-5, max_iters: int = 4096, wet_res: int = 64, spray_cap: int = 1024) -> WorldHeader:
    """A header for a scene of `blocks` (x, y, z) 4^3 blocks of cell size `h_cell` from `origin`."""
    ref = _reference_params()
    h = WorldHeader()
    h.magic, h.version = WORLD_MAGIC, WORLD_VERSION
    h.n_particles, h.n_verts, h.n_tris, h.n_vtri = n_particles, n_verts, n_tris, n_vtri
    h.n_shots, h.n_blocks_prev, h.n_spray, h.wet_res = 0, n_blocks_prev, 0, wet_res
    h.spray_cap, h.block_cap = spray_cap, block_cap
    h.iters, h.substeps, h.air_substeps = iters, substeps, air_substeps
    h.unconverged, h.started, h.max_iters = 0, 1, max_iters
    h.t = h.t_start = h.t0 = 0.0
    h.dx = h_cell
    p = h.params
    p.origin[:] = [origin[0], origin[1], origin[2], h_cell]
    p.dims[:] = [4 * blocks[0], 4 * blocks[1], 4 * blocks[2], n_particles]
    p.bdims[:] = [blocks[0], blocks[1], blocks[2], block_cap]
    p.gravity[:] = [gravity[0], gravity[1], gravity[2], sound_speed]
    p.fluid[:] = [1000.0, 0.8, dt_max, 0.5 * h_cell]
    p.wet[:] = [ref.wet[0], 0.0, 0.0, 0.0]
    p.limits[:] = [wet_res, spray_cap, iters, 0]
    p.solve[:] = [solve_tol, 0.0, 0.0, 0.0]
    p.mem[:] = [n_verts, substeps, air_substeps, 0]
    p.rubber[:] = list(ref.rubber)
    p.rubber2[:] = list(ref.rubber2)
    # The knot's solid plug, out of the domain.
    p.knot[:] = [origin[0] - 1.0, origin[1] - 1.0, origin[2] - 1.0, 0.0]
    s = h.state
    s.n_blocks_prev = n_blocks_prev
    s.mem_dt = s.cap_dt = s.air_dt = FLT_MAX
    return h


def particles(pos: np.ndarray, vel=None, pressure=None, alive=None) -> np.ndarray:
    """The PARTICLES section: 20 floats a particle (position w = 1, velocity w = alive, affine
    terms zero, c0.w = carried pressure in Pa)."""
    n = len(pos)
    p = np.zeros((n, 20), np.float32)
    p[:, :3] = pos
    p[:, 3] = 1.0
    if vel is not None:
        p[:, 4:7] = vel
    p[:, 7] = 1.0 if alive is None else alive
    if pressure is not None:
        p[:, 11] = pressure
    return p


def lattice(lo_cells, hi_cells, h_cell: float, origin) -> np.ndarray:
    """Positions of 2 x 2 x 2 particles per cell (at 1/4 and 3/4 of the cell per axis) over the
    cells lo..hi-1, as the scene builder's lattice without its jitter."""
    ax = [(np.arange(2 * lo, 2 * hi) + 0.5) * 0.5 * h_cell + origin[k] for k, (lo, hi) in enumerate(zip(lo_cells, hi_cells))]
    g = np.meshgrid(*ax, indexing="ij")
    return np.stack([a.reshape(-1) for a in g], 1).astype(np.float32)


def no_membrane(pos) -> dict:
    """One massless vertex, no triangles: the rubber's kernels skip it."""
    return {"MEM_X": np.array([[pos[0], pos[1], pos[2], 0.0]], np.float32), "VTRI_OFF": np.zeros(2, np.uint32)}


def all_blocks(blocks) -> np.ndarray:
    """Every block slot of the domain, ascending (slot = (x * by + y) * bz + z)."""
    return np.arange(blocks[0] * blocks[1] * blocks[2], dtype=np.uint32)


def cell_coords(block_list: np.ndarray, blocks) -> np.ndarray:
    """Domain cell coordinates (x, y, z) of every cell of the listed blocks, in storage order
    (64 cells a block, local index x * 16 + y * 4 + z)."""
    bx, by, bz = blocks
    s = block_list.astype(np.int64)
    b = np.stack([s // (bz * by), (s // bz) % by, s % bz], 1)
    li = np.arange(64)
    l = np.stack([li // 16, (li // 4) % 4, li % 4], 1)
    return (b[:, None, :] * 4 + l[None, :, :]).reshape(-1, 3)
