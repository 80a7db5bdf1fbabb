"""Synthetic tissues and the epi5_MT cell-file format.

A tissue is one epi5_MT CellManager worth of particles in the reference's
index layout (epi5_MT/cellmanager.h:87-91): membrane particles (state MEMB)
first, then dermis (DER), then every other cell. Membrane particle j sits at
lattice column j % nmx, row j // nmx, which is the wiring _memb_init assumes
(epi5_MT/cellmanager.cpp:114-166, square branch).

Positions are jittered with splitmix64 so that the same seed gives the same
doubles in numpy, in C and on the GPU host. Text I/O follows the reference
loader's column order (epi5_MT/cellmanager.cpp:243-244); doubles are written
with 17 significant digits so the reference's %lf parse restores them exactly.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

# Cell states, epi5_MT/define.h:36-47.
ALIVE, DEAD, DISA, UNUSED, FIX, BLANK, DER, MUSUME, AIR, MEMB = range(10)
SQUARE, TRIANGULAR = 0, 1  # membrane lattices

R_MAX = 1.4     # define.h:116
R_DER = 1.4     # define.h:119
R_MEMB = 1.0    # define.h:122

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64_uniform(seed: int, count: int, start: int = 0) -> np.ndarray:
    """`count` uniforms in [0,1) from splitmix64 draws start+1 ... start+count."""
    with np.errstate(over="ignore"):
        k = np.arange(start + 1, start + count + 1, dtype=np.uint64)
        s = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + _GOLDEN * k
        z = (s ^ (s >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def mix_seed(*parts: int) -> int:
    """Derive a 64-bit seed from integers (splitmix64 finaliser chain)."""
    h = 0x243F6A8885A308D3
    for p in parts:
        with np.errstate(over="ignore"):
            u = splitmix64_uniform((h ^ (p & 0xFFFFFFFFFFFFFFFF)) & 0xFFFFFFFFFFFFFFFF, 1)[0]
        h = int(u * 2.0**53) ^ ((h << 7) & 0xFFFFFFFFFFFFFFFF)
    return h & 0xFFFFFFFFFFFFFFFF


@dataclass
class Params:
    """Force-law constants; defaults are epi5_MT's compile-time values
    (epi5_MT/cell_interaction.cpp:21-45, define.h:86,116-135)."""
    dt: float = 0.01
    eps_m: float = 0.01
    p_memb: float = 1.0 / 4          # 1 / COMPRESS_FACTOR
    der_der_const: float = 0.2
    k_total: float = 3.0
    k_desmosome: float = 3.0 * 0.01  # K_TOTAL * K_DESMOSOME_RATIO
    kspring: float = 25.0
    kspring_d: float = 5.0
    kbend: float = 0.5
    delta_r: float = 0.4 * R_DER
    para_ljp2: float = 0.005
    kspring_division: float = 5.0
    lj_thresh: float = 1.2
    thresh_sp: float = 3.0

    def scaled(self, spring: float = 1.0, eps: float = 1.0, bend: float = 1.0) -> "Params":
        """Every spring constant times `spring`, eps_m times `eps`, KBEND times `bend`."""
        p = Params(**self.__dict__)
        p.der_der_const *= spring
        p.k_total *= spring
        p.k_desmosome *= spring
        p.kspring *= spring
        p.kspring_d *= spring
        p.kspring_division *= spring
        p.eps_m *= eps
        p.kbend *= bend
        return p

    def as_tuple(self):
        return (self.dt, self.eps_m, self.p_memb, self.der_der_const, self.k_total,
                self.k_desmosome, self.kspring, self.kspring_d, self.kbend, self.delta_r,
                self.para_ljp2, self.kspring_division, self.lj_thresh, self.thresh_sp)


@dataclass
class Tissue:
    nmx: int
    nmy: int
    lx: float
    ly: float
    lz: float
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    radius: np.ndarray
    state: np.ndarray                 # uint8
    agek: np.ndarray
    spr_nat_len: np.ndarray
    pair: np.ndarray                  # int32, -1 = none
    rest_div_times: np.ndarray        # int32
    nmemb: int = 0
    nder: int = 0
    params: Params = field(default_factory=Params)
    name: str = ""
    # ageb (division age) of each cell: used only by the reference's state
    # renewal (cell_state_renew.cpp), never by the mechanics; None = all 0
    ageb: Optional[np.ndarray] = None
    # membrane lattice: SQUARE (4 links, TRI_MEMB undefined) or TRIANGULAR
    # (6 links, the reference's default TRI_MEMB build); nmy counts rows
    lattice: int = 0

    @property
    def n(self) -> int:
        return int(self.x.shape[0])

    def copy(self) -> "Tissue":
        t = Tissue(self.nmx, self.nmy, self.lx, self.ly, self.lz,
                   self.x.copy(), self.y.copy(), self.z.copy(), self.radius.copy(),
                   self.state.copy(), self.agek.copy(), self.spr_nat_len.copy(),
                   self.pair.copy(), self.rest_div_times.copy(), self.nmemb, self.nder,
                   Params(**self.params.__dict__), self.name,
                   None if self.ageb is None else self.ageb.copy(), self.lattice)
        return t

    def validate(self) -> None:
        n = self.n
        for a in (self.y, self.z, self.radius, self.state, self.agek, self.spr_nat_len,
                  self.pair, self.rest_div_times):
            assert a.shape == (n,)
        assert self.nmemb == self.nmx * self.nmy
        assert np.all(self.state[: self.nmemb] == MEMB)
        assert np.all(self.state[self.nmemb: self.nmemb + self.nder] == DER)
        assert not np.any(self.state[self.nmemb + self.nder:] == MEMB)
        assert not np.any(self.state[self.nmemb + self.nder:] == DER)

    # ---- reference text format (epi5_MT/cellmanager.cpp:198-323) ----
    def write_reference_file(self, path: str) -> None:
        lines = []
        for i in range(self.n):
            lines.append(
                "%d %d %r %r %r %r %r %r %r %r %d %r %r %d %r %d %d" % (
                    i, int(self.state[i]), float(self.radius[i]),
                    0.0 if self.ageb is None else float(self.ageb[i]), float(self.agek[i]),
                    0.0, float(self.x[i]), float(self.y[i]), float(self.z[i]), 0.0,
                    int(self.rest_div_times[i]), 0.0, 0.0, 0, float(self.spr_nat_len[i]),
                    int(self.pair[i]), -1))
        with open(path, "w") as f:
            f.write("\n".join(lines) + "\n")


def _wrap(v: np.ndarray, L: float) -> np.ndarray:
    v = np.where(v < 0.0, v + L, v)
    return np.where(v >= L, v - L, v)


def layered_tissue(side: int, layers: int, seed: int, *, spacing: float = 1.0,
                   cell_radius: float = 0.5, memb_z: float = 1.0, first_layer_z: float = 2.0,
                   jitter: float = 0.1, lz: float = 32.0, params: Optional[Params] = None,
                   name: str = "") -> Tissue:
    """Square membrane of side x side particles under `layers` jittered layers of
    ALIVE cells, periodic side*spacing box in x and y.

    Membrane particle (j, k) sits at ((j+0.5)s, (k+0.5)s, memb_z); cell (i, j, l)
    at (i s, j s, first_layer_z + l s) plus U(-jitter, +jitter) on each axis, so
    every cell sits over the centre of a membrane square.
    """
    L = side * spacing
    nm = side * side
    nc = layers * side * side
    jj, kk = np.meshgrid(np.arange(side), np.arange(side), indexing="xy")
    mx = ((jj.ravel() + 0.5) * spacing).astype(np.float64)
    my = ((kk.ravel() + 0.5) * spacing).astype(np.float64)
    mz = np.full(nm, memb_z)
    ll, cj, ci = np.meshgrid(np.arange(layers), np.arange(side), np.arange(side), indexing="ij")
    u = splitmix64_uniform(seed, 3 * nc).reshape(nc, 3)
    jit = (2.0 * u - 1.0) * jitter
    cx = _wrap(ci.ravel() * spacing + jit[:, 0], L)
    cy = _wrap(cj.ravel() * spacing + jit[:, 1], L)
    cz = first_layer_z + ll.ravel() * spacing + jit[:, 2]
    n = nm + nc
    t = Tissue(
        nmx=side, nmy=side, lx=L, ly=L, lz=lz,
        x=np.concatenate([mx, cx]), y=np.concatenate([my, cy]), z=np.concatenate([mz, cz]),
        radius=np.concatenate([np.full(nm, R_MEMB), np.full(nc, cell_radius)]),
        state=np.concatenate([np.full(nm, MEMB, np.uint8), np.full(nc, ALIVE, np.uint8)]),
        agek=np.zeros(n), spr_nat_len=np.zeros(n), pair=np.full(n, -1, np.int32),
        rest_div_times=np.zeros(n, np.int32), nmemb=nm, nder=0,
        params=params or Params(), name=name)
    t.validate()
    return t


def tri_layered_tissue(nmx: int, rows: int, layers: int, seed: int, *, spacing: float = 1.0,
                       cell_radius: float = 0.5, memb_z: float = 1.0, first_layer_z: float = 2.0,
                       jitter: float = 0.1, lz: float = 32.0, params: Optional[Params] = None,
                       name: str = "") -> Tissue:
    """Triangular membrane (the reference's default TRI_MEMB lattice,
    cellmanager.cpp:70-111) of nmx x rows particles under `layers` jittered
    layers of ALIVE cells on the same lattice. Site (j, k) sits at
    ((j + 0.5 (k mod 2)) s, k s sqrt(3)/2): even rows' diagonal neighbours are
    j-1 and j, odd rows' j and j+1, as the reference wires them; the box is
    nmx s by rows s sqrt(3)/2 (rows even, so the lattice is periodic)."""
    assert rows % 2 == 0
    dy = spacing * math.sqrt(3.0) / 2.0
    lx, ly = nmx * spacing, rows * dy
    nm = nmx * rows
    jj, kk = np.meshgrid(np.arange(nmx), np.arange(rows), indexing="xy")
    sx = ((jj.ravel() + 0.5 * (kk.ravel() % 2)) * spacing).astype(np.float64)
    sy = (kk.ravel() * dy + 0.25 * dy).astype(np.float64)
    nc = layers * nm
    u = splitmix64_uniform(seed, 3 * nc).reshape(nc, 3) if nc else np.zeros((0, 3))
    jit = (2.0 * u - 1.0) * jitter
    lay = np.repeat(np.arange(layers), nm)
    cx = _wrap(np.tile(sx, layers) + jit[:, 0], lx)
    cy = _wrap(np.tile(sy, layers) + jit[:, 1], ly)
    cz = first_layer_z + lay * spacing + jit[:, 2]
    n = nm + nc
    t = Tissue(
        nmx=nmx, nmy=rows, lx=lx, ly=ly, lz=lz,
        x=np.concatenate([sx, cx]), y=np.concatenate([sy, cy]),
        z=np.concatenate([np.full(nm, memb_z), cz]),
        radius=np.concatenate([np.full(nm, R_MEMB), np.full(nc, cell_radius)]),
        state=np.concatenate([np.full(nm, MEMB, np.uint8), np.full(nc, ALIVE, np.uint8)]),
        agek=np.zeros(n), spr_nat_len=np.zeros(n), pair=np.full(n, -1, np.int32),
        rest_div_times=np.zeros(n, np.int32), nmemb=nm, nder=0,
        params=params or Params(), name=name, lattice=TRIANGULAR)
    t.validate()
    return t


def config1(seed: int = 0) -> Tissue:
    """16x16 membrane, 512 cells in 2 layers, periodic 16x16 box (plain FP64 drop-in case)."""
    return layered_tissue(16, 2, seed, name="C1")


def config2(seed: int = 1) -> Tissue:
    """64x64 membrane, 32,768 cells in 8 layers, periodic 64x64 box."""
    return layered_tissue(64, 8, seed, name="C2")


def config3(seed: int = 2) -> Tissue:
    """256x256 membrane, 1,048,576 cells in 16 layers, periodic 256x256 box."""
    return layered_tissue(256, 16, seed, name="C3")


C4_SIDES = (16, 24, 32, 48, 64)


def config4_specs(seed: int = 3, n_tissues: int = 512) -> List[tuple]:
    """Per tissue of the ensemble: (side, layers, params), without positions.
    Side uniform in {16,24,32,48,64}, layers uniform in 2..8, accepted when
    layers*side^2 is in [2048, 40000]; spring, LJ epsilon and bending scale
    each log-uniform in [0.5, 2]. A tissue has side^2 membrane particles and
    layers*side^2 cells."""
    out = []
    for t in range(n_tissues):
        s = mix_seed(seed, t)
        draw = 0
        while True:
            u = splitmix64_uniform(s, 2, start=draw)
            draw += 2
            side = C4_SIDES[min(int(u[0] * len(C4_SIDES)), len(C4_SIDES) - 1)]
            layers = 2 + min(int(u[1] * 7), 6)
            if 2048 <= layers * side * side <= 40000:
                break
        sc = splitmix64_uniform(s, 3, start=draw)
        scale = np.exp(np.log(0.5) + sc * (np.log(2.0) - np.log(0.5)))
        p = Params().scaled(spring=float(scale[0]), eps=float(scale[1]), bend=float(scale[2]))
        out.append((side, layers, p))
    return out


def config4(seed: int = 3, n_tissues: int = 512,
            indices: Optional[Sequence[int]] = None) -> List[Tissue]:
    """Ensemble of independent tissues (config4_specs); `indices` selects
    which of the n_tissues to generate (default: all), so a rank can build
    only its own shard. Tissue t is the same whatever n_tissues is."""
    specs = config4_specs(seed, n_tissues)
    if indices is None:
        indices = range(n_tissues)
    return [layered_tissue(specs[t][0], specs[t][1], mix_seed(seed, t, 1), params=specs[t][2],
                           name=f"C4[{t}]") for t in indices]


def tri_rows(side: int, spacing: float = 1.0) -> int:
    """An even row count near `side` for a triangular membrane whose box
    (rows * spacing * sqrt(3) / 2 in y) the reference's grid covers: it has
    (int)(LY / 2 + 0.5) bins of 2.0 (cell_connection.cpp:22-26), so LY must
    not round down."""
    for rows in range(side + side % 2, side + 32, 2):
        ly = rows * spacing * math.sqrt(3.0) / 2.0
        if int(ly / 2.0 + 0.5) * 2.0 >= ly:
            return rows
    raise ValueError("no row count found")


def config4_tri(seed: int = 3, n_tissues: int = 512,
                indices: Optional[Sequence[int]] = None) -> List[Tissue]:
    """The ensemble of config4 with triangular membranes (TRI_MEMB, the
    reference's default lattice): same sides, layers and constants, rows =
    tri_rows(side), cells on the same lattice."""
    specs = config4_specs(seed, n_tissues)
    if indices is None:
        indices = range(n_tissues)
    return [tri_layered_tissue(specs[t][0], tri_rows(specs[t][0]), specs[t][1],
                               mix_seed(seed, t, 1), params=specs[t][2], name=f"C4T[{t}]")
            for t in indices]


def config5(seed: int = 4) -> Tissue:
    """Adjoint case: config-2 geometry (64x64 membrane, 32,768 cells)."""
    return layered_tissue(64, 8, seed, name="C5")


def mixed_state_tissue(seed: int = 7, lattice: int = SQUARE) -> Tissue:
    """Small tissue exercising every force law of the path: dermis (DER) under a
    32-wide membrane at the reference's natural 0.5 spacing, stem (FIX) cells
    paired with daughters (MUSUME), unpaired MUSUME with divisions left, and
    ALIVE / DEAD / AIR cells above, some older than THRESH_SP. The layout
    follows the reference's own initial-state generator
    (epi_intg/calc/init_gen.cpp:46-104): DER lattice at pitch 2 R_der, membrane
    at Z_LEVEL + R_memb, FIX at R_max + R_memb + Z_LEVEL + R_memb. The
    membrane is a 32 x 32 square lattice in a 16 x 16 box, or (TRIANGULAR)
    32 x 36 rows of the reference's default triangular lattice, rows
    0.5 sqrt(3)/2 apart, in a 16 x 15.59 box."""
    L = 16.0
    side = 32
    pitch = 0.5
    z_level = 2.0 * R_DER
    if lattice == TRIANGULAR:
        rows = 36
        dy = pitch * math.sqrt(3.0) / 2.0
        LY = rows * dy
        nm = side * rows
        jj, kk = np.meshgrid(np.arange(side), np.arange(rows), indexing="xy")
        mx = (jj.ravel() + 0.5 * (kk.ravel() % 2)) * pitch
        my = kk.ravel() * dy + 0.25 * dy
    else:
        rows = side
        LY = L
        nm = side * side
        jj, kk = np.meshgrid(np.arange(side), np.arange(side), indexing="xy")
        mx = (jj.ravel() + 0.5) * pitch
        my = (kk.ravel() + 0.5) * pitch
    xs = [list(mx)]
    ys = [list(my)]
    zs = [[z_level + R_MEMB] * nm]
    rs = [[R_MEMB] * nm]
    st = [[MEMB] * nm]
    ag = [[0.0] * nm]
    sp = [[0.0] * nm]
    pr = [[-1] * nm]
    rd = [[0] * nm]
    nder_side = int(L / (2.0 * R_DER))
    for k in range(nder_side):
        for j in range(nder_side):
            xs.append([R_DER + 2.0 * j * R_DER]); ys.append([R_DER + 2.0 * k * R_DER])
            zs.append([R_DER]); rs.append([R_DER]); st.append([DER]); ag.append([0.0])
            sp.append([0.0]); pr.append([-1]); rd.append([0])
    nder = nder_side * nder_side
    u = splitmix64_uniform(seed, 4096)
    ui = iter(u)

    def jit(a=0.15):
        return (2.0 * next(ui) - 1.0) * a

    others = []  # (state, x, y, z, r, agek, rest_div, pair_slot, spr)
    fix_z = R_MAX + R_MEMB + z_level + R_MEMB
    # four FIX cells on a circle; the first two each paired with a MUSUME
    for l in range(4):
        cx = L / 2 + (L / 4) * math.cos(2 * math.pi * l / 4) + jit()
        cy = L / 2 + (L / 4) * math.sin(2 * math.pi * l / 4) + jit()
        others.append([FIX, cx, cy, fix_z + jit(0.05), R_MAX, 0.0, 15, None, 0.0])
        if l < 2:
            others.append([MUSUME, cx + 2.6 + jit(0.05), cy + jit(0.05), fix_z + jit(0.05), R_MAX,
                           0.0, 3, len(others) - 1, 2.5])
            others[-2][7] = len(others) - 1
            others[-2][8] = 2.5
    # unpaired MUSUME cells, with and without remaining divisions
    for l, rest in enumerate((2, 0, 1)):
        others.append([MUSUME, 1.5 + 4.5 * l + jit(), 1.5 + jit(), fix_z + jit(0.05), R_MAX,
                       0.0, rest, None, 0.0])
    # an ALIVE pair (divided earlier), to exercise the pair spring between non-stem cells
    others.append([ALIVE, 4.0 + jit(), 4.0 + jit(), fix_z + 2.7 + jit(0.05), R_MAX, 1.0, 0, None, 2.6])
    others.append([ALIVE, 6.7 + jit(), 4.0 + jit(), fix_z + 2.7 + jit(0.05), R_MAX, 1.0, 0,
                   len(others) - 1, 2.6])
    others[-2][7] = len(others) - 1
    # suprabasal layers: ALIVE, then DEAD / AIR on top; every second one old
    k = 0
    for layer, state in ((1, ALIVE), (2, DEAD), (3, AIR)):
        for iy in range(3):
            for ix in range(3):
                if layer == 1 and iy == 0 and ix < 2:
                    continue  # room for the ALIVE pair
                others.append([state, 2.8 + 4.2 * ix + jit(), 2.8 + 4.2 * iy + jit(),
                               fix_z + 2.7 * layer + jit(0.05), R_MAX,
                               4.0 if (k % 2) else 0.5, 0, None, 0.0])
                k += 1
    base = nm + nder
    for o in others:
        xs.append([o[1] % L]); ys.append([o[2] % LY]); zs.append([o[3]]); rs.append([o[4]])
        st.append([o[0]]); ag.append([o[5]]); rd.append([o[6]])
        pr.append([-1 if o[7] is None else base + o[7]]); sp.append([o[8]])
    cat = lambda a, dt: np.array([v for part in a for v in part], dtype=dt)
    t = Tissue(nmx=side, nmy=rows, lx=L, ly=LY, lz=32.0,
               x=cat(xs, np.float64), y=cat(ys, np.float64), z=cat(zs, np.float64),
               radius=cat(rs, np.float64), state=cat(st, np.uint8), agek=cat(ag, np.float64),
               spr_nat_len=cat(sp, np.float64), pair=cat(pr, np.int32),
               rest_div_times=cat(rd, np.int32), nmemb=nm, nder=nder,
               name="mixed" if lattice == SQUARE else "mixed_tri", lattice=lattice)
    t.validate()
    return t


def renewal_tissue(seed: int = 7) -> Tissue:
    """mixed_state_tissue with ages set so that the reference's state renewal
    (cell_state_renew.cpp:400-433) acts within the first steps: the two
    unpaired FIX cells and the unpaired MUSUME with divisions left are past
    their division age (cell_divide, :227-279; with a division draw that
    passes they divide and the batch grows), the old DEAD cells are past
    ADHE_CONST with few connections (removed, :330-345, which reorders the
    cell array), and one ALIVE cell is at THRESH_DEAD (cornified, :347-361)."""
    t = mixed_state_tissue(seed)
    ageb = np.zeros(t.n)
    cells = np.arange(t.nmemb + t.nder, t.n)
    fix = cells[t.state[cells] == FIX]
    ageb[fix[t.pair[fix] < 0]] = 100.0
    mus = cells[(t.state[cells] == MUSUME) & (t.pair[cells] < 0) & (t.rest_div_times[cells] > 0)]
    ageb[mus] = 5.0
    dead = cells[t.state[cells] == DEAD]
    t.agek[dead[::2]] = 40.0
    alive = cells[(t.state[cells] == ALIVE) & (t.pair[cells] < 0)]
    t.agek[alive[0]] = 22.0
    t.ageb = ageb
    t.name = "renewal"
    t.validate()
    return t


def field_tissue(seed: int = 7, lattice: int = SQUARE) -> Tissue:
    """mixed_state_tissue with cell ages inside the window where the
    external-stimulus source is on (ext_stim.cpp:8-16: an ALIVE or DEAD cell
    with THRESH_DEAD - 0.5 < agek <= THRESH_DEAD + 2): every other DEAD cell
    at 22.5 and two ALIVE cells at 21.8, so the diffusion has sources."""
    t = mixed_state_tissue(seed, lattice)
    cells = np.arange(t.nmemb + t.nder, t.n)
    dead = cells[t.state[cells] == DEAD]
    t.agek[dead[::2]] = 22.5
    alive = cells[(t.state[cells] == ALIVE) & (t.pair[cells] < 0)]
    t.agek[alive[:2]] = 21.8
    t.name = "field"
    t.validate()
    return t


def read_reference_file(path: str, nmx: int, lx: float, ly: float, lz: float,
                        lattice: int = TRIANGULAR, name: str = "") -> Tissue:
    """Loads an epi5_MT initial-state file (the format of its cman_init
    loader, cellmanager.cpp:198-330: id, state, radius, ageb, agek, ca2p, x,
    y, z, ca2p_avg, rest_div_times, ex_fat, in_fat, touch, spr_nat_len,
    pair id, stem id; reading stops at the first BLANK cell). nmx is the
    membrane's row length (define.h NMX); the membrane rows are
    nmemb / nmx."""
    rows = []
    with open(path) as f:
        for line in f:
            v = line.split()
            if not v:
                continue
            if int(v[1]) == BLANK:
                break
            rows.append(v)
    n = len(rows)
    st = np.array([int(r[1]) for r in rows], np.uint8)
    col = lambda k: np.array([float(r[k]) for r in rows], np.float64)
    nmemb = int((st == MEMB).sum())
    nder = int((st == DER).sum())
    pair = np.array([int(r[15]) for r in rows], np.int32)
    pair[pair < 0] = -1
    t = Tissue(nmx=nmx, nmy=nmemb // nmx, lx=lx, ly=ly, lz=lz, x=col(6), y=col(7), z=col(8),
               radius=col(2), state=st, agek=col(4), spr_nat_len=col(14), pair=pair,
               rest_div_times=np.array([int(r[10]) for r in rows], np.int32), nmemb=nmemb,
               nder=nder, name=name or path, ageb=col(3), lattice=lattice)
    return t


def read_reference_frames(path: str):
    """Parse oracle frames (positions, sorted CSR connections, dermis) as
    written by the oracle harnesses. Returns a list of dicts."""
    data = open(path, "rb").read()
    off = 0
    frames = []
    while off < len(data):
        tag, step, n = np.frombuffer(data, np.int32, 3, off)
        assert tag == 0x454D5246, "bad frame tag"
        off += 12
        x = np.frombuffer(data, np.float64, n, off); off += 8 * n
        y = np.frombuffer(data, np.float64, n, off); off += 8 * n
        z = np.frombuffer(data, np.float64, n, off); off += 8 * n
        co = np.frombuffer(data, np.int32, n + 1, off); off += 4 * (n + 1)
        ci = np.frombuffer(data, np.int32, int(co[-1]), off); off += 4 * int(co[-1])
        de = np.frombuffer(data, np.int32, n, off); off += 4 * n
        frames.append(dict(step=int(step), x=x.copy(), y=y.copy(), z=z.copy(),
                           conn_off=co.copy(), conn_idx=ci.copy(), dermis=de.copy()))
    return frames
