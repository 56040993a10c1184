"""REV lattice scenes as flat arrays, in the layout of ``vx_scene_desc``.

``Scene`` mirrors the fields of the reference's ``Scene`` (src/scene.rs:309-351)
and ``Voxel`` (src/voxel.rs:7-21) that the elastic solve reads. The builders
follow ``Scene::from_voxels`` (src/scene.rs:445-573) and ``Scene::new``
(src/scene.rs:1572-1721). The synthetic workloads (10^3 wood cube, 64^3 mixed
block, 160^3 damaged lattice, batched boxes) are generated from seeds.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import materials as M

EMPTY = 0xFFFFFFFF
CELL32 = np.float32(0.01)
CELL = float(CELL32)
ROOM_TEMPERATURE = 293.15


@dataclass
class Scene:
    n: int
    cells: np.ndarray            # (n,3) int32 lattice coordinates
    position: np.ndarray         # (n,3) float64
    rotation: np.ndarray         # (n,4) float64 xyzw
    kinematic: np.ndarray        # (n,) uint8
    mass: np.ndarray             # (n,) float32
    material: np.ndarray         # (n,) uint32 index into materials
    materials: list              # list[materials.Material]
    fiber: np.ndarray            # (n,3) float32 body-frame fibre axis
    anisotropy: np.ndarray       # (n,) float32
    solid_fraction: np.ndarray   # (n,) float32
    thermal_strength: np.ndarray # (n,) float32
    thermal_delta: np.ndarray    # (n,) float32  T - T_reference
    neighbor: np.ndarray         # (3,n) uint32 axis-major
    formation_offset: np.ndarray # (3,n,3) float32
    plastic_strain: np.ndarray   # (3,n,3) float32
    damage: np.ndarray           # (3,n) float32
    equivalent_plastic: np.ndarray = None  # (3,n) float32
    velocity: np.ndarray = None  # (n,3) float64
    target_mask: np.ndarray = None  # (n,) uint8 bit a = axis a targeted
    target: np.ndarray = None    # (n,3) float64
    loads: np.ndarray = None     # (n,3) float64 applied loads (N)
    meta: dict = field(default_factory=dict)

    def __post_init__(self):
        n = self.n
        if self.equivalent_plastic is None:
            self.equivalent_plastic = np.zeros((3, n), np.float32)
        if self.velocity is None:
            self.velocity = np.zeros((n, 3), np.float64)
        if self.target_mask is None:
            self.target_mask = np.zeros(n, np.uint8)
        if self.target is None:
            self.target = np.zeros((n, 3), np.float64)
        if self.loads is None:
            self.loads = np.zeros((n, 3), np.float64)

    # -- derived views -------------------------------------------------------
    def material_records(self) -> np.ndarray:
        return M.records(self.materials)

    def free_mask(self) -> np.ndarray:
        """(n,3) 0/1 free axes (src/solver.rs:1554-1565)."""
        fixed = np.zeros((self.n, 3), bool)
        fixed |= self.kinematic.astype(bool)[:, None]
        for a in range(3):
            fixed[:, a] |= ((self.target_mask >> a) & 1).astype(bool)
        return (~fixed).astype(np.float64)

    def active_count(self) -> int:
        return int((self.free_mask().sum(axis=1) > 0).sum())

    def bond_count(self) -> int:
        return int((self.neighbor != EMPTY).sum())

    def fix_voxels(self, idx) -> None:
        """Scene::fix_voxels (src/scene.rs:895-930): kinematic after topology is built."""
        self.kinematic[np.asarray(idx)] = 1
        self.velocity[np.asarray(idx)] = 0.0

    def set_axis_targets(self, idx, values, axes=(0, 1, 2)) -> None:
        idx = np.asarray(idx)
        for a in axes:
            self.target_mask[idx] |= np.uint8(1 << a)
            self.target[idx, a] = np.asarray(values)[..., a] if np.ndim(values) else values

    def copy(self) -> "Scene":
        out = Scene(**{k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in self.__dict__.items()})
        out.materials = list(self.materials)
        out.meta = dict(self.meta)
        return out


# ---------------------------------------------------------------------------
def build_topology(cells: np.ndarray, kinematic: np.ndarray) -> np.ndarray:
    """neighbor[axis, i] = REV at cells[i] + e_axis when both REVs share the
    kinematic flag, else EMPTY (src/scene.rs:558-570)."""
    cells = np.asarray(cells, np.int64)
    n = len(cells)
    nbr = np.full((3, n), EMPTY, np.uint32)
    if n == 0:
        return nbr
    lo = cells.min(axis=0)
    ext = cells.max(axis=0) - lo + 2
    vol = int(ext[0]) * int(ext[1]) * int(ext[2])
    rel = cells - lo
    if vol <= 64 * max(n, 1_000_000):
        grid = np.full(vol, -1, np.int64)
        key = (rel[:, 2] * ext[1] + rel[:, 1]) * ext[0] + rel[:, 0]
        grid[key] = np.arange(n)
        for a in range(3):
            r2 = rel.copy()
            r2[:, a] += 1
            k2 = (r2[:, 2] * ext[1] + r2[:, 1]) * ext[0] + r2[:, 0]
            j = grid[k2]
            ok = j >= 0
            ok[ok] &= kinematic[j[ok]] == kinematic[ok]
            nbr[a, ok] = j[ok].astype(np.uint32)
    else:  # sparse lattice: dictionary lookup
        occ = {tuple(c): i for i, c in enumerate(cells.tolist())}
        for i, c in enumerate(cells.tolist()):
            for a in range(3):
                c2 = list(c)
                c2[a] += 1
                j = occ.get(tuple(c2))
                if j is not None and kinematic[j] == kinematic[i]:
                    nbr[a, i] = j
    return nbr


def _positions_f32(cells: np.ndarray) -> np.ndarray:
    # key * CELL + CELL/2 evaluated in f32 (src/scene.rs:1589-1592, :110-113)
    c = cells.astype(np.float32)
    p = (c * CELL32).astype(np.float32) + np.float32(CELL32 * np.float32(0.5))
    return p.astype(np.float32).astype(np.float64)


def _unit(v) -> np.ndarray:
    v = np.asarray(v, np.float32)
    return (v / np.float32(np.sqrt(np.float32(np.dot(v, v))))).astype(np.float32)


def from_cells(cells, material_ids, materials_table, *, kinematic=None, fiber=None,
               anisotropy=None, temperature=ROOM_TEMPERATURE, bond_kinematic=None) -> Scene:
    """Scene::from_voxels (src/scene.rs:445-573) for REVs on integer cells.

    ``bond_kinematic`` is the kinematic flag the topology sees (defaults to
    ``kinematic``); pass zeros to build one body and fix REVs afterwards, as
    Scene::fix_voxels does.
    """
    cells = np.asarray(cells, np.int32).reshape(-1, 3)
    n = len(cells)
    mid = np.asarray(material_ids, np.uint32).reshape(-1)
    if mid.size == 1 and n != 1:
        mid = np.full(n, mid[0], np.uint32)
    kin = np.zeros(n, np.uint8) if kinematic is None else np.asarray(kinematic, np.uint8).copy()
    bk = kin if bond_kinematic is None else np.asarray(bond_kinematic, np.uint8)
    fib = np.tile(np.array([0, 0, 1], np.float32), (n, 1)) if fiber is None else np.asarray(fiber, np.float32).reshape(n, 3)
    ani = np.zeros(n, np.float32) if anisotropy is None else np.broadcast_to(np.asarray(anisotropy, np.float32), (n,)).copy()
    dens = np.array([m.density for m in materials_table], np.float32)
    mass = (dens[mid] * np.float32(CELL32 ** 3)).astype(np.float32)
    cell3 = np.float32(CELL32 * CELL32 * CELL32)
    mass = (dens[mid] * cell3).astype(np.float32)
    temps = np.broadcast_to(np.asarray(temperature, np.float64), (n,))
    solid = np.array([materials_table[m].solid_fraction(t) for m, t in zip(mid, temps)], np.float32) if n else np.zeros(0, np.float32)
    therm = np.array([materials_table[m].thermal_strength_scale(t) for m, t in zip(mid, temps)], np.float32) if n else np.zeros(0, np.float32)
    s = Scene(
        n=n,
        cells=cells,
        position=_positions_f32(cells),
        rotation=np.tile(np.array([0, 0, 0, 1], np.float64), (n, 1)),
        kinematic=kin,
        mass=mass,
        material=mid,
        materials=list(materials_table),
        fiber=fib,
        anisotropy=ani,
        solid_fraction=solid,
        thermal_strength=therm,
        thermal_delta=np.zeros(n, np.float32),
        neighbor=build_topology(cells, bk),
        formation_offset=np.zeros((3, n, 3), np.float32),
        plastic_strain=np.zeros((3, n, 3), np.float32),
        damage=np.zeros((3, n), np.float32),
    )
    return s


def scene_new(dimensions, *, branch=(0, 0, 0), ground=(0, 0, 0), fibers=(0.0, 0.0, 1.0),
              anisotropy=1.0, materials_table=None) -> Scene:
    """Scene::new layout (src/scene.rs:1572-1721): a wood trunk centred in x/y,
    an optional branch and a kinematic stone ground below it."""
    table = M.table() if materials_table is None else materials_table
    nx, ny, nz = dimensions
    keys, mats, ani, fib, kin = [], [], [], [], []
    seen = set()
    fiber = _unit(fibers)

    def add(key, comp, a, fixed, f):
        if key in seen:
            return
        seen.add(key)
        keys.append(key)
        mats.append(comp)
        ani.append(a)
        fib.append(f)
        kin.append(1 if fixed else 0)

    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                add((x - nx // 2, y - ny // 2, z), 1, anisotropy, False, fiber)
    bx, by, bz = branch
    for z in range(bz):
        for y in range(by):
            for x in range(bx):
                add((nx // 2 + x, y - by // 2, nz * 2 // 3 + z), 1, anisotropy, False,
                    np.array([1, 0, 0], np.float32))
    gx, gy, gz = ground
    for z in range(gz):
        for y in range(gy):
            for x in range(gx):
                add((x - gx // 2, y - gy // 2, -z - 1), 3, 0.0, True, np.array([0, 0, 1], np.float32))
    cells = np.array(keys, np.int32).reshape(-1, 3)
    return from_cells(cells, np.array(mats), table, kinematic=np.array(kin, np.uint8),
                      fiber=np.array(fib, np.float32).reshape(-1, 3), anisotropy=np.array(ani, np.float32))


def wood_config_materials(young=12e9, young_perp=0.3e9, shear=0.75e9, density=600.0):
    """Wood with the moduli and density the workloads state; the other fields
    (strengths, fracture energies, modes) are the built-in wood row."""
    from dataclasses import replace
    t = M.table()
    t[1] = replace(t[1], young=young, young_perp=young_perp, shear=shear, density=density)
    return t


def grid_cells(nx, ny, nz, origin=(0, 0, 0)) -> np.ndarray:
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    c = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1).astype(np.int32)
    return c + np.asarray(origin, np.int32)


# ---------------------------------------------------------------------------
# Synthetic workloads
# ---------------------------------------------------------------------------
def wood_cube(edge=10, displacement=1e-4) -> Scene:
    """10x10x10 wood cube: grain +Z, E 12/0.3 GPa, G 0.75 GPa, 600 kg/m^3.
    Bottom layer kinematic (fixed after bonding), top layer targeted at
    rest + (0, 0, displacement) on all axes."""
    table = wood_config_materials()
    cells = grid_cells(edge, edge, edge)
    s = from_cells(cells, 1, table, anisotropy=1.0)
    s.fix_voxels(np.nonzero(cells[:, 2] == 0)[0])
    top = np.nonzero(cells[:, 2] == edge - 1)[0]
    s.target_mask[top] = 7
    s.target[top] = s.position[top] + np.array([0.0, 0.0, displacement])
    s.meta.update(workload="wood_cube", edge=edge, dt=1e-3, substeps=1, gravity=(0, 0, 0),
                  passes=1, tolerance=1e-10)
    return s


def impose_axis_targets(scene: Scene) -> Scene:
    """Move every targeted axis of every REV onto its target, as the substep's
    prediction does before the solve (src/solver.rs:506-512). On the wood cube
    this lifts the top layer by the displacement, so the pass that follows
    loads the bonds below it (the axial fixture of src/experiments.rs:79-85)."""
    for a in range(3):
        sel = ((scene.target_mask >> a) & 1).astype(bool)
        scene.position[sel, a] = scene.target[sel, a]
    return scene


def predict_from_rest(scene: Scene, h: float, gravity) -> np.ndarray:
    """Predicted positions of the first substep from rest (v0 = 0): the explicit
    prediction of src/solver.rs:500-523. Free REVs drift by g h^2 on their
    untargeted axes; targeted axes sit on their targets; kinematic REVs stay."""
    g = np.asarray(gravity, np.float64)
    v = np.zeros_like(scene.position)
    free = scene.kinematic == 0
    v[free] = g * h
    for a in range(3):
        v[((scene.target_mask >> a) & 1).astype(bool), a] = 0.0
    x = scene.position + v * h
    for a in range(3):
        m = ((scene.target_mask >> a) & 1).astype(bool)
        x[m, a] = scene.target[m, a]
    return x


def random_unit_vectors(rng, n) -> np.ndarray:
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v.astype(np.float32)


def mixed_block(edge=64, seed=1) -> Scene:
    """64^3 block, material uniform per REV over wood (12/0.3 GPa, grain a
    random unit vector per REV), iron 200 GPa, stone 50 GPa, aluminium 70 GPa;
    bottom layer fixed; gravity -9.81."""
    from dataclasses import replace
    rng = np.random.default_rng(seed)
    table = wood_config_materials()
    table[5] = replace(table[5], young=70e9, young_perp=70e9)
    cells = grid_cells(edge, edge, edge)
    n = len(cells)
    choice = np.array([1, 2, 3, 5], np.uint32)[rng.integers(0, 4, n)]
    fib = np.tile(np.array([0, 0, 1], np.float32), (n, 1))
    wood = choice == 1
    fib[wood] = random_unit_vectors(rng, int(wood.sum()))
    ani = np.where(wood, 1.0, 0.0).astype(np.float32)
    s = from_cells(cells, choice, table, fiber=fib, anisotropy=ani)
    s.fix_voxels(np.nonzero(cells[:, 2] == 0)[0])
    s.meta.update(workload="mixed_block", edge=edge, dt=1e-3, substeps=1, gravity=(0, 0, -9.81),
                  passes=5, tolerance=1e-8, seed=seed)
    return s


def damaged_lattice(edge=160, seed=2, removed=0.10, force_sigma=0.05) -> Scene:
    """160^3 wood lattice, grain Z, 10% of bonds removed uniformly at random,
    persistent per-REV forces N(0, 0.05 N) on free REVs; bottom layer fixed."""
    rng = np.random.default_rng(seed)
    table = wood_config_materials()
    cells = grid_cells(edge, edge, edge)
    s = from_cells(cells, 1, table, anisotropy=1.0)
    bonded = np.nonzero(s.neighbor.reshape(-1) != EMPTY)[0]
    drop = rng.choice(bonded, size=int(round(removed * len(bonded))), replace=False)
    flat = s.neighbor.reshape(-1)
    flat[drop] = EMPTY
    s.fix_voxels(np.nonzero(cells[:, 2] == 0)[0])
    free = s.kinematic == 0
    s.loads[free] = rng.normal(0.0, force_sigma, size=(int(free.sum()), 3))
    s.meta.update(workload="damaged_lattice", edge=edge, dt=1e-3, substeps=1, gravity=(0, 0, 0),
                  passes=8, tolerance=1e-8, seed=seed)
    return s


def box_union_scene(rng, edge_lo=8, edge_hi=48, max_boxes=4, displacement=5e-5) -> Scene:
    """One batched-workload scene: a random union of 1-4 axis-aligned boxes in a
    cube whose edge is log-uniform over [edge_lo, edge_hi]; one random material
    and grain; the x=min face clamped and the x=max face targeted
    +displacement along +x."""
    from dataclasses import replace
    edge = int(round(math.exp(rng.uniform(math.log(edge_lo), math.log(edge_hi)))))
    occ = np.zeros((edge, edge, edge), bool)
    for _ in range(int(rng.integers(1, max_boxes + 1))):
        a = rng.integers(0, edge, 3)
        b = rng.integers(0, edge, 3)
        lo, hi = np.minimum(a, b), np.maximum(a, b) + 1
        # boxes span the clamped axis so every scene is held
        lo[0], hi[0] = 0, edge
        occ[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = True
    x, y, z = np.nonzero(occ)
    cells = np.stack([x, y, z], axis=1).astype(np.int32)
    order = np.lexsort((cells[:, 0], cells[:, 1], cells[:, 2]))
    cells = cells[order]
    table = wood_config_materials()
    table[5] = replace(table[5], young=70e9, young_perp=70e9)
    comp = int(np.array([1, 2, 3, 5])[rng.integers(0, 4)])
    g = random_unit_vectors(rng, 1)[0]
    n = len(cells)
    s = from_cells(cells, comp, table, fiber=np.tile(g, (n, 1)), anisotropy=1.0 if comp == 1 else 0.0)
    s.fix_voxels(np.nonzero(cells[:, 0] == 0)[0])
    far = np.nonzero(cells[:, 0] == edge - 1)[0]
    s.target_mask[far] = 7
    s.target[far] = s.position[far] + np.array([displacement, 0.0, 0.0])
    s.meta.update(workload="box_union", edge=edge, dt=1e-3, substeps=1, gravity=(0, 0, 0),
                  passes=1, tolerance=1e-8)
    return s
