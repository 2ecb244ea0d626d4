"""Generates tests/golden/lj_golden.npz: golden vectors for the CPU oracle.

A second, independent restatement of the reference algorithms, written in
numpy and plain Python from the reference sources (cited per function), run
on the same inputs the reference's own tests use. tests/test_golden.py checks
the C oracle (oracle/) and the CUDA library's host helpers against it.

    python tests/golden/make_golden.py
"""

import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MASK = (1 << 64) - 1
F = np.float32


def xorshift_stream(seed):
    """lennard_jones.rs:1410-1415: uniform in (0, 1)."""
    s = seed

    def nxt():
        nonlocal s
        s ^= (s << 13) & MASK
        s ^= s >> 7
        s ^= (s << 17) & MASK
        return ((s >> 11) + 0.5) / float(1 << 53)

    return nxt


def lattice_sites(count, size, sites, temperature, seed):
    """lennard_jones.rs:1401-1441."""
    gap = [size[k] / sites[k] for k in range(3)]
    rnd = xorshift_stream(seed | 1)

    def gaussian():
        r = math.sqrt(-2.0 * math.log(rnd()))
        return r * math.cos(6.283185307179586 * rnd())

    pos = np.zeros((count, 3))
    vel = np.zeros((count, 3))
    for i in range(count):
        c = [i % sites[0], (i // sites[0]) % sites[1], i // (sites[0] * sites[1])]
        for k in range(3):
            pos[i, k] = (c[k] + 0.5) * gap[k]
        for k in range(3):
            vel[i, k] = gaussian() * math.sqrt(temperature)
    for k in range(3):
        s = 0.0
        for i in range(count):
            s += vel[i, k]
        mean = s / count
        vel[:, k] -= mean
    return pos, vel


def lattice(count, box, temperature, seed):
    """lennard_jones.rs:1379-1382."""
    per_side = math.ceil(math.cbrt(count))
    return lattice_sites(count, [box] * 3, [per_side] * 3, temperature, seed)


def round_half_away(x):
    """f64::round for x >= 0: halves go up."""
    r = math.floor(x)
    return int(r + 1) if x - r >= 0.5 else int(r)


def lattice_box(count, size, temperature, seed):
    """lennard_jones.rs:1388-1399 (ties go to the later axis, as Rust's max_by)."""
    spacing = math.cbrt(size[0] * size[1] * size[2] / count)
    sites = [max(1, round_half_away(l / spacing)) for l in size]
    while sites[0] * sites[1] * sites[2] < count:
        widest = 0
        for k in (1, 2):
            if not (size[widest] / sites[widest] > size[k] / sites[k]):
                widest = k
        sites[widest] += 1
    return lattice_sites(count, size, sites, temperature, seed)


def jitter(pos, seed=99):
    """tests/thermodynamics.rs:61-69 and tests/coexistence.rs:81-88."""
    s = seed
    out = pos.copy()
    for i in range(len(out)):
        for k in range(3):
            s ^= (s << 13) & MASK
            s ^= s >> 7
            s ^= (s << 17) & MASK
            out[i, k] += ((s >> 11) / float(1 << 53) - 0.5) * 0.3
    return out


def pcg_seed(seed, i):
    """lennard_jones.rs:584-592."""
    z = ((seed << 32) | i) & MASK
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
    return (z ^ (z >> 31)) & 0xFFFFFFFF


def pcg_next(state):
    """lennard_jones.wgsl:168-173; returns (output, new state)."""
    s = (state * 747796405 + 2891336453) & 0xFFFFFFFF
    word = ((((s >> ((s >> 28) + 4)) ^ s) & 0xFFFFFFFF) * 277803737) & 0xFFFFFFFF
    return ((word >> 22) ^ word) & 0xFFFFFFFF, s


def f32_bits(x):
    return int(np.array([x], F).view(np.uint32)[0])


def bits_f32(b):
    return np.array([b], np.uint32).view(F)[0]


def last_bit(h):
    """lennard_jones.wgsl:128-131."""
    e = (f32_bits(h) >> 23) & 0xFF
    return bits_f32((max(e, 24) - 23) << 23)


def pack_lo(hi, lo):
    """lennard_jones.wgsl:135-142."""
    bits = 0x20000000
    for k in range(3):
        t = F(lo[k]) / last_bit(hi[k])
        t = min(max(t, F(-0.5)), F(0.5))
        q = int(np.rint(F(t) * F(510.0)))
        bits |= (q + 256) << (9 * k)
    return bits


def unpack_lo(h, bits, k):
    """lennard_jones.wgsl:144-152."""
    q = F(((bits >> (9 * k)) & 511) - 256)
    return F(q / F(510.0)) * last_bit(h)


def setup(n, vel, box, cutoff, skin):
    """lennard_jones.rs:450-474, 507-515 (the parts the rebuild needs)."""
    box_f = [F(b) for b in box]
    radius = cutoff + skin
    cells = [int(math.floor(float(b) / radius)) for b in box_f]
    assert min(cells) >= 3
    cell_size = [F(float(box_f[k]) / cells[k]) for k in range(3)]
    volume = float(box_f[0]) * float(box_f[1]) * float(box_f[2])
    expected = 4.0 / 3.0 * math.pi * radius ** 3 * (n / volume)
    capacity = math.ceil(2.0 * expected + 32.0)
    return dict(box_f=box_f, cells=cells, cell_size=cell_size, capacity=capacity,
                list_r2=F(radius * radius))


def rebuild(s, pos, reorder):
    """grid.wgsl:11-148 then lennard_jones.wgsl:421-499, in f32 as written."""
    n = len(pos)
    hi = pos.astype(F)
    lo = (pos - hi.astype(np.float64)).astype(F)
    nx, ny, nz = s["cells"]

    def cell_of(h):
        c = []
        for k in range(3):
            v = int(np.floor(F(h[k]) / s["cell_size"][k]))
            c.append(min(max(v, 0), s["cells"][k] - 1))
        return (c[2] * ny + c[1]) * nx + c[0]

    cell = [cell_of(hi[i]) for i in range(n)]
    members = [[] for _ in range(nx * ny * nz)]
    for i in range(n):
        members[cell[i]].append(i)
    start = [0]
    for m in members:
        start.append(start[-1] + len(m))
    order = [i for m in members for i in m]
    ids = list(range(n))
    if reorder:
        hi, lo = hi[order], lo[order]
        pos = pos[order]
        cell = [cell[i] for i in order]
        ids = order
        order = list(range(n))
    packed = [pack_lo(hi[i], lo[i]) for i in range(n)]
    lists = []
    for i in range(n):
        ci = cell[i]
        cc = (ci % nx, (ci // nx) % ny, ci // (nx * ny))
        found = []
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    c = (((cc[2] + dz) % nz) * ny + (cc[1] + dy) % ny) * nx + (cc[0] + dx) % nx
                    for t in range(start[c], start[c + 1]):
                        j = order[t]
                        if j == i:
                            continue
                        d = []
                        for k in range(3):
                            a = F(hi[j, k] - hi[i, k])
                            b = F(unpack_lo(hi[j, k], packed[j], k) - lo[i, k])
                            e = F(a + b)
                            side = s["box_f"][k]
                            d.append(F(e - F(side * np.rint(F(e / side)))))
                        r2 = F(F(F(d[0] * d[0]) + F(d[1] * d[1])) + F(d[2] * d[2]))
                        if r2 < s["list_r2"]:
                            found.append(j)
        lists.append(found)
    return dict(ids=np.array(ids, np.uint32), cell=np.array(cell, np.uint32),
                start=np.array(start, np.uint32), order=np.array(order, np.uint32),
                lists=lists, packed=np.array(packed, np.uint32))


def main():
    out = {}
    # tests/thermodynamics.rs:60-69: jittered lattice(1000, 11, 1, 3)
    p, v = lattice(1000, 11.0, 1.0, 3)
    out["lattice_pos"], out["lattice_vel"] = p, v
    out["jittered_cube"] = jitter(p)
    # tests/coexistence.rs:79-91: jittered lattice_box(1000, [9, 10.5, 14.25], 1, 3)
    pb, vb = lattice_box(1000, [9.0, 10.5, 14.25], 1.0, 3)
    out["box_pos"], out["box_vel"] = pb, vb
    out["jittered_box"] = jitter(pb)
    # tests/heat.rs:92-96: liquid(9 x 9 x 12) = lattice_box(round(0.8442 V), ., 1, 11)
    count = round_half_away(0.8442 * 9 * 9 * 12)
    out["liquid_pos"], out["liquid_vel"] = lattice_box(count, [9.0, 9.0, 12.0], 1.0, 11)
    # random streams
    out["pcg_seed"] = np.array([pcg_seed(s, i) for s in (1, 3, 7) for i in range(16)], np.uint32)
    seq = []
    for st in (1, 12345, 0xDEADBEEF):
        for _ in range(8):
            o, st = pcg_next(st)
            seq.append(o)
    out["pcg_sequence"] = np.array(seq, np.uint32)
    # packed positions of the jittered cube, wrapped as LennardJones::new does
    L = float(F(11.0))
    wrapped = np.mod(out["jittered_cube"], L)
    s = setup(1000, v, [11.0] * 3, 2.5, 0.3)
    r = rebuild(s, wrapped, reorder=True)
    out["rebuild_ids"], out["rebuild_cell"], out["rebuild_start"] = r["ids"], r["cell"], r["start"]
    out["rebuild_packed"] = r["packed"]
    out["rebuild_counts"] = np.array([len(x) for x in r["lists"]], np.uint32)
    out["rebuild_lists"] = np.concatenate([np.array(x, np.uint32) for x in r["lists"]])
    out["rebuild_capacity"] = np.array([s["capacity"]], np.uint32)
    np.savez_compressed(os.path.join(HERE, "lj_golden.npz"), **out)
    print("wrote", os.path.join(HERE, "lj_golden.npz"))


if __name__ == "__main__":
    main()
