"""Autotuner for how the force kernels read the Verlet list.

The list rows staged in shared memory and the L1 that serves the neighbour
gathers share each SM's 256 KB, so the tile depth (rows per tile, tiles in
flight) trades list-stream latency against gather hit rate; the rows can also
stream per thread from global memory without L1 allocation (no tiles). This builds one
library per candidate into build/tune/ (git-ignored), times the step kernel on
a workload in a child process per variant (CUDA events around every launch,
L2 flushed between steps), and prints the ranking as JSON lines. Needs a GPU.

    python virial-engine_b200/tune.py [--cells 40] [--steps 60]

The winner's settings become the defaults of VLJ_LIST_STREAM / VLJ_L1_CARVEOUT
(csrc/vlj_internal.cuh, csrc/vlj_forces.cu) or VLJ_TILE_ROWS / VLJ_TILE_SLOTS.

    python virial-engine_b200/tune.py --kernel build [--cells 40] [--steps 30]

times the list build's variants instead (candidates per round, staged
candidates per warp, blocks per SM, two home particles per test:
VLJ_BUILD_* in csrc/vlj_build.cu) by the wall time of a forced rebuild.

    python virial-engine_b200/tune.py --kernel tiles [--cells 40] [--steps 40]

times the step kernel with cell tiles (VLJ_TILES=1) against the per-particle
gathers: bricks per x-row 3, 4, 5, 6, 8 (the tile size and the threads per
block follow from it; VLJ_TILE_COLS at run time) for the encoded-word tiles,
f32 offsets from the brick centre (VLJ_TILE_F32) and the next row read ahead
(VLJ_TILE_PIPE).
"""

import argparse
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "build", "tune")
# name -> preprocessor overrides: rows streamed without L1 allocation under
# shared-memory carve-out hints (percent), or the TMA tile ring (rows per tile,
# tiles in flight)
# list-build variants: the test's loop order (home particles or candidate
# groups outermost), candidates staged per warp, and the blocks per SM the
# registers are sized for
BUILD_CANDIDATES = {
    "groups_outer_stage512_b6": {},
    "groups_outer_stage448_b6": {"VLJ_BUILD_STAGE": 448},
    "groups_outer_stage416_b7": {"VLJ_BUILD_STAGE": 416, "VLJ_BUILD_BLOCKS_PER_SM": 7},
    "groups_outer_stage352_b8": {"VLJ_BUILD_STAGE": 352, "VLJ_BUILD_BLOCKS_PER_SM": 8},
    "homes_outer_stage512_b6": {"VLJ_BUILD_ORDER": 1},
    "homes_outer_stage416_b7": {"VLJ_BUILD_ORDER": 1, "VLJ_BUILD_STAGE": 416,
                                "VLJ_BUILD_BLOCKS_PER_SM": 7},
}
# cell-tile variants: compile-time form x bricks per x-row (0: tiles off)
TILE_CANDIDATES = {
    "encoded": {},
    "f32": {"VLJ_TILE_F32": 1},
    "read_ahead": {"VLJ_TILE_PIPE": 1},
}
TILE_COLS = (0, 3, 4, 5, 6, 8)
CANDIDATES = {
    "stream_c0": {"VLJ_LIST_STREAM": 1, "VLJ_L1_CARVEOUT": 0},
    "stream_c4": {"VLJ_LIST_STREAM": 1, "VLJ_L1_CARVEOUT": 4},
    "stream_c8": {"VLJ_LIST_STREAM": 1, "VLJ_L1_CARVEOUT": 8},
    "stream_c4_remap": {"VLJ_LIST_STREAM": 1, "VLJ_L1_CARVEOUT": 4, "VLJ_STEP_REMAP": 1},
    "stream_c8_remap": {"VLJ_LIST_STREAM": 1, "VLJ_L1_CARVEOUT": 8, "VLJ_STEP_REMAP": 1},
    "ahead_c4": {"VLJ_LIST_STREAM": 1, "VLJ_GATHER_AHEAD": 1, "VLJ_L1_CARVEOUT": 4},
    "tma_r1_s4": {"VLJ_LIST_STREAM": 0, "VLJ_TILE_ROWS": 1, "VLJ_TILE_SLOTS": 4},
}


def child(lib, cells, steps, cols=None):
    os.environ["VLJ_LIBRARY"] = lib
    if cols is not None:
        os.environ["VLJ_TILES"] = "1" if cols else "0"
        if cols:
            os.environ["VLJ_TILE_COLS"] = str(cols)
    sys.path.insert(0, HERE)
    import torch
    import virial_lj as vl
    p, box = vl.lattice_fcc(cells, 0.8442, 1.0, 7)
    stream = torch.cuda.Stream()
    sim = vl.LennardJones(p, vl.Settings([box] * 3, dt=0.005, shifted_force=True,
                                         thermostat=vl.Langevin(1.0, 1.0, 7)),
                          stream=stream.cuda_stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    sim.step(10)
    sim.kernel_timing(True)
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        sim.step(1)
    ms, n = sim.kernel_time()
    print(json.dumps({"step_kernel_us": ms * 1e3 / n, "launches": n,
                      "tiles": list(sim.tile_info())}))


def build_child(lib, cells, rebuilds):
    """Wall time of a forced rebuild (decide, the grid, the list build; the
    stream waited on), averaged: the list build is most of it."""
    os.environ["VLJ_LIBRARY"] = lib
    sys.path.insert(0, HERE)
    import time
    import virial_lj as vl
    p, box = vl.lattice_fcc(cells, 0.8442, 1.0, 7)
    sim = vl.LennardJones(p, vl.Settings([box] * 3, dt=0.005, shifted_force=True,
                                         thermostat=vl.Langevin(1.0, 1.0, 7)))
    sim.run(20)
    sim.force_rebuild()
    t0 = time.perf_counter()
    for _ in range(rebuilds):
        sim.force_rebuild()
    us = (time.perf_counter() - t0) / rebuilds * 1e6
    print(json.dumps({"rebuild_us": us, "rebuilds": rebuilds}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cells", type=int, default=40)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--child", default=None)
    ap.add_argument("--kernel", choices=["step", "build", "tiles"], default="step",
                    help="tune the force kernels' list reading (step), the list build, or "
                         "the cell-tile step kernel against the gathers (tiles)")
    ap.add_argument("--cols", type=int, default=None, help=argparse.SUPPRESS)
    ap.add_argument("--no-build", action="store_true",
                    help="time the variants already in build/tune (built elsewhere)")
    ap.add_argument("--build-only", action="store_true", help="build the variants, time nothing")
    args = ap.parse_args()
    if args.child:
        if args.kernel == "build":
            build_child(args.child, args.cells, args.steps)
        else:
            child(args.child, args.cells, args.steps, args.cols)
        return
    sys.path.insert(0, HERE)
    import build
    os.makedirs(OUT_DIR, exist_ok=True)
    results = []
    candidates = {"build": BUILD_CANDIDATES, "tiles": TILE_CANDIDATES}.get(args.kernel, CANDIDATES)
    key = "rebuild_us" if args.kernel == "build" else "step_kernel_us"
    for name, defines in candidates.items():
        lib = os.path.join(OUT_DIR, f"libvirial_lj_{name}.so")
        if not args.no_build:
            build.build(defines=defines, out=lib, force=True)
        if args.build_only:
            continue
        for cols in (TILE_COLS if args.kernel == "tiles" else (None,)):
            if args.kernel == "tiles" and cols == 0 and name != "encoded":
                continue  # tiles off: the same kernel in every variant
            cmd = [sys.executable, __file__, "--child", lib, "--cells", str(args.cells),
                   "--steps", str(args.steps), "--kernel", args.kernel]
            if cols is not None:
                cmd += ["--cols", str(cols)]
            out = subprocess.run(cmd, capture_output=True, text=True)
            if out.returncode != 0:
                print(json.dumps({"variant": name, "error": out.stderr[-500:]}), flush=True)
                continue
            r = json.loads(out.stdout.strip().splitlines()[-1])
            r.update(variant=name if cols is None else f"{name}_cols{cols}", defines=defines)
            results.append(r)
            print(json.dumps(r), flush=True)
    if results:
        best = min(results, key=lambda r: r[key])
        print(json.dumps({"best": best}))


if __name__ == "__main__":
    main()
