"""Initial particle scenes.

Reference scenes replicate the reference's host lattice loops with FP32
accumulation of the loop variable, exactly as its float loop counters do:
  ref_box_3d2   SPHSystem::add_box_particle    SPH-3D-2/sph_system.cpp:247-264
  ref_new_3d2   SPHSystem::add_new_particle    SPH-3D-2/sph_system.cpp:266-283
  ref_box_3d4   SPHSystem::add_box_particle    SPH-3D-4/sph_system.cpp:248-289
  ref_sphere_3d4 SPHSystem::add_new_particle   SPH-3D-4/sph_system.cpp:291-332
  ref_init_2d   SPHSystem::add_init_particle   SPH-2D/sph_system.cpp:148-162
The SI dam-break scenes are lattice blocks at spacing s, each coordinate
jittered by U(-0.01 s, +0.01 s) drawn from a SplitMix64 counter stream keyed
by (seed, particle index, axis), so every scene is reproducible on any host.
"""
import numpy as np

f32 = np.float32


def _frange(start, step, cond):
    """Float32 loop `for (x = start; cond(x); x += step)`."""
    out = []
    x = f32(start)
    step = f32(step)
    while cond(x):
        out.append(x)
        x = f32(x + step)
    return out


def _grid(xs, ys, zs=None):
    # reference loop order: x outer, y, z inner
    if zs is None:
        return np.array([(x, y) for x in xs for y in ys], dtype=np.float32)
    return np.array([(x, y, z) for x in xs for y in ys for z in zs], dtype=np.float32)


def ref_box_3d2(cfg):
    h = f32(cfg.kernel[0])
    W, H, L = (f32(cfg.world[a]) for a in range(3))
    half = f32(h / f32(2.0))
    step = f32(h * f32(0.8))
    xs = _frange(half, step, lambda x: x <= f32(W / f32(2)))
    ys = _frange(half, step, lambda y: f32(H - y) >= half)
    zs = _frange(half, step, lambda z: f32(L - z) >= half)
    pos = _grid(xs, ys, zs)
    return pos, np.zeros_like(pos), np.ones(len(pos), np.uint32)


def ref_new_3d2(cfg):
    hl, hs = f32(cfg.kernel[0]), f32(cfg.kernel[1])
    W, H, L = (f32(cfg.world[a]) for a in range(3))
    half = f32(hl / f32(2.0))
    start = f32(half + f32(4))
    step = f32(hs * f32(0.4))
    xs = _frange(start, step, lambda x: f32(f32(W - f32(4)) - x) >= half)
    ys = _frange(start, step, lambda y: f32(f32(H - f32(4)) - y) >= half)
    zs = _frange(start, step, lambda z: f32(f32(L - f32(4)) - z) >= half)
    pos = _grid(xs, ys, zs)
    return pos, np.zeros_like(pos), np.full(len(pos), 2, np.uint32)


def ref_box_3d4(cfg):
    sp = f32(cfg.kernel[1])
    W, H, L = (f32(cfg.world[a]) for a in range(3))
    step = f32(sp * f32(0.5))
    xs = _frange(sp, step, lambda x: f32(W - x) >= sp)
    ys = _frange(sp, step, lambda y: y < f32(H / f32(4)))
    zs = _frange(sp, step, lambda z: f32(L - z) >= sp)
    pos = _grid(xs, ys, zs)
    return pos, np.zeros_like(pos), np.full(len(pos), 2, np.uint32)


def ref_sphere_3d4(cfg):
    """The falling sphere of SPH-3D-4 without the reference's double count
    (add_particle already increments m_num_particle, :324 increments again,
    leaving every other record uninitialised)."""
    r = f32(10.0)
    spacing = f32(float(cfg.kernel[1]) * 0.5)
    pts = []
    z = -r
    while z <= r:
        y = -r
        while y <= r:
            x = -r
            while x <= r:
                l = np.sqrt(f32(f32(f32(x * x) + f32(y * y)) + f32(z * z)), dtype=np.float32)
                if l <= f32(5.0):
                    pts.append((f32(24.0) + x, f32(18.0) + y, f32(12.0) + z))
                x = f32(x + spacing)
            y = f32(y + spacing)
        z = f32(z + spacing)
    pos = np.array(pts, dtype=np.float32)
    vel = np.zeros_like(pos)
    vel[:, 1] = -10.0
    return pos, vel, np.full(len(pos), 2, np.uint32)


def ref_init_2d(cfg):
    rl, hl = f32(cfg.radius[0]), f32(cfg.kernel[0])
    W, D = f32(cfg.world[0]), f32(cfg.world[1])
    half = f32(rl / f32(2.0))
    step = f32(hl * f32(0.5))
    xs = _frange(half, step, lambda x: x < f32(W / f32(2)))
    ys = _frange(half, step, lambda y: f32(D - y) >= half)
    pos = _grid(xs, ys)
    return pos, np.zeros_like(pos), np.ones(len(pos), np.uint32)


# ---------------------------------------------------------------- SI scenes
_M64 = (1 << 64) - 1


def splitmix64(x):
    """SplitMix64 finaliser over uint64 numpy arrays (Steele et al., 2014)."""
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(_M64)
    z = x
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & np.uint64(_M64)
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & np.uint64(_M64)
    return z ^ (z >> np.uint64(31))


def uniform(seed, index, stream):
    """U[0,1) doubles for counters `index` of stream `stream` under `seed`."""
    key = (np.uint64(seed) * np.uint64(0x100000001B3)) ^ (np.uint64(stream) << np.uint64(40))
    with np.errstate(over="ignore"):
        bits = splitmix64(np.asarray(index, np.uint64) ^ key)
    return (bits >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))


def lattice(counts, spacing, origin, seed, first_index=0, jitter=0.01):
    """Block of prod(counts) particles at (i + 0.5) * spacing + origin, each
    axis jittered by U(-jitter*s, +jitter*s); x outer, z inner."""
    d = len(counts)
    idx = np.indices(counts).reshape(d, -1).T.astype(np.float64)
    pos = origin + (idx + 0.5) * spacing
    ids = np.arange(len(pos), dtype=np.uint64) + np.uint64(first_index)
    for a in range(d):
        u = uniform(seed, ids, a)
        pos[:, a] += (2.0 * u - 1.0) * jitter * spacing
    return pos.astype(np.float32)


def dam_2d(cfg, seed=0):
    """64 x 64 block at s = 0.01 in the lower-left quarter of the 1.28 box."""
    pos = lattice((64, 64), 0.01, np.zeros(2), seed)
    return pos, np.zeros_like(pos), np.ones(len(pos), np.uint32)


def dam_3d2(cfg, seed=0):
    """64 x 64 x 32 block at s = 0.01 in the 1.28 x 0.64 x 0.64 box."""
    pos = lattice((64, 64, 32), 0.01, np.zeros(3), seed)
    return pos, np.zeros_like(pos), np.ones(len(pos), np.uint32)


def sphere_points(count, spacing, centre):
    """The `count` lattice points (spacing s) nearest to the centre, in
    increasing distance (ties by lattice order)."""
    r = int(np.ceil((count * 3.0 / (4.0 * np.pi)) ** (1.0 / 3.0))) + 2
    g = np.arange(-r, r + 1, dtype=np.float64)
    pts = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    d2 = (pts * pts).sum(1)
    order = np.argsort(d2, kind="stable")[:count]
    return centre + pts[order] * spacing


def dam_3d4(cfg, seed=0, sphere=65536):
    """128 x 128 x 64 block at s = 0.005 plus a 65 536-particle sphere at the
    same spacing (radius ~0.125) centred 0.18 above the block top, falling at
    (0, -2, 0)."""
    s = 0.005
    block = lattice((128, 128, 64), s, np.zeros(3), seed)
    parts = [block]
    vels = [np.zeros_like(block)]
    if sphere:
        centre = np.array([0.32, 0.64 + 0.18, 0.16])
        sp = sphere_points(sphere, s, centre)
        ids = np.arange(len(sp), dtype=np.uint64) + np.uint64(len(block))
        for a in range(3):
            sp[:, a] += (2.0 * uniform(seed, ids, a) - 1.0) * 0.01 * s
        sp = sp.astype(np.float32)
        v = np.zeros_like(sp)
        v[:, 1] = -2.0
        parts.append(sp)
        vels.append(v)
    pos = np.concatenate(parts)
    return pos, np.concatenate(vels), np.ones(len(pos), np.uint32)


def block_3d(cfg, counts=(32, 32, 32), spacing=0.01, seed=0):
    pos = lattice(counts, spacing, np.zeros(3), seed)
    return pos, np.zeros_like(pos), np.ones(len(pos), np.uint32)


def batch_scenes(cfg, count, seed=0, n_min=1024, n_max=65536, gap_cells=2, subset=None):
    """`count` independent dam-break scenes packed into one world for a
    batched handle (sph_set_scenes).

    Scene k draws, from the SplitMix64 streams of `seed`: a particle count
    log-uniform in [n_min, n_max]; a block aspect ratio with each axis
    factor log-uniform in [1/2, 2] (normalised to product 1); viscosity
    log-uniform in [1e-3, 1e-1]; gas stiffness uniform in [1, 5].  The block
    is a jittered lattice at spacing s = kernel[0] / 2 in the low corner of
    its box; the box is twice the block along x, 1.5 times its height along
    y and (3D) one cell deeper than the block along z, rounded up to whole
    cells.  Boxes sit at whole-cell offsets, `gap_cells` apart, packed in
    shelves over the x-z plane (3D) or the x-y plane (2D).

    `subset` (a list of scene numbers) packs only those scenes, each drawn
    exactly as in the full set (e.g. one rank's share of a sharded batch).

    Returns (cfg, boxes, pos, vel, level, scene, counts): cfg is a copy with
    world, ncell and max_particle (4x the particles) set; boxes is a list of
    (lo, hi, viscosity, gas_constant) for Solver.set_scenes; particles are
    scene by scene in scene order (scene index = position in the subset)."""
    dim = int(cfg.dim)
    s = float(cfg.kernel[0]) * 0.5
    cs = float(cfg.cell_size)
    k = np.arange(count, dtype=np.uint64)
    u_n = uniform(seed, k, 16)
    n_target = np.exp(np.log(n_min) + u_n * (np.log(n_max) - np.log(n_min)))
    asp = np.stack([2.0 ** (2.0 * uniform(seed, k, 17 + a) - 1.0) for a in range(dim)], 1)
    asp /= np.prod(asp, axis=1, keepdims=True) ** (1.0 / dim)
    mu = np.exp(np.log(1e-3) + uniform(seed, k, 21) * (np.log(1e-1) - np.log(1e-3)))
    stiff = 1.0 + 4.0 * uniform(seed, k, 22)
    blocks = np.maximum(4, np.rint(n_target[:, None] ** (1.0 / dim) * asp)).astype(np.int64)
    first_of = np.concatenate([[0], np.cumsum(np.prod(blocks, axis=1))])   # jitter ids as in the full set
    if subset is not None:
        subset = np.asarray(subset, np.int64)
        blocks, mu, stiff, first_of = blocks[subset], mu[subset], stiff[subset], first_of[subset]
        count = len(subset)
    # box extents in cells
    ext = np.zeros((count, dim), np.int64)
    ext[:, 0] = np.ceil(2.0 * blocks[:, 0] * s / cs - 1e-9)
    ext[:, 1] = np.ceil(1.5 * blocks[:, 1] * s / cs - 1e-9)
    if dim == 3:
        ext[:, 2] = np.ceil(blocks[:, 2] * s / cs - 1e-9) + 1
    # shelf packing: shelves run along x, stack along the last axis; in 3D
    # every box spans y from 0
    sec = dim - 1
    g = gap_cells
    width = int(max(np.sqrt(((ext[:, 0] + g) * (ext[:, sec] + g)).sum()) * 1.25, ext[:, 0].max() + g))
    order = np.argsort(-ext[:, sec], kind="stable")
    off = np.zeros((count, dim), np.int64)
    cx = cz = depth = 0
    for i in order:
        if cx > 0 and cx + ext[i, 0] > width:
            cz += depth + g
            cx = depth = 0
        off[i, 0] = cx
        off[i, sec] = cz
        cx += ext[i, 0] + g
        depth = max(depth, int(ext[i, sec]))
    top = off + ext
    out = cfg.copy()
    for a in range(dim):
        out.ncell[a] = int(top[:, a].max())
        out.world[a] = f32(out.ncell[a]) * f32(cs)
    if dim == 2:
        out.ncell[2] = 1
        out.world[2] = 0.0
    boxes, parts, scene = [], [], []
    for i in range(count):
        lo = [f32(off[i, a]) * f32(cs) for a in range(dim)]
        hi = [f32(top[i, a]) * f32(cs) for a in range(dim)]
        boxes.append((lo, hi, float(f32(mu[i])), float(f32(stiff[i]))))
        p = lattice(tuple(int(b) for b in blocks[i]), s, np.array(lo, np.float64), seed,
                    first_index=int(first_of[i]))
        parts.append(p)
        scene.append(np.full(len(p), i, np.uint32))
    pos = np.concatenate(parts)
    counts = np.array([len(p) for p in parts], np.int64)
    out.max_particle = int(4 * len(pos))
    return (out, boxes, pos, np.zeros_like(pos), np.ones(len(pos), np.uint32),
            np.concatenate(scene), counts)
