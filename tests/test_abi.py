"""The C ABI library loads and exports every function include/virial_lj.h
declares; host-only entry points work without a GPU."""

import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    text = open(os.path.join(ROOT, "include", "virial_lj.h")).read()
    return sorted(set(re.findall(r"VLJ_API\s+[\w\s\*]+?\b(vlj_\w+)\s*\(", text)))


def test_header_declares_the_api():
    names = declared()
    for must in ["vlj_create", "vlj_destroy", "vlj_step", "vlj_run", "vlj_measure", "vlj_poll",
                 "vlj_measure_now", "vlj_read_particles", "vlj_sample_profile",
                 "vlj_read_profile", "vlj_record_heat_current", "vlj_read_heat_current",
                 "vlj_set_temperature", "vlj_lattice", "vlj_lattice_box", "vlj_batch_create",
                 "vlj_batch_step"]:
        assert must in names


def test_library_exports_every_declared_symbol(vl):
    import ctypes
    lib = ctypes.CDLL(vl.library_path())
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_library_hides_internal_symbols(vl):
    out = os.popen(f"nm -D --defined-only {vl.library_path()}").read()
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert exported <= set(declared()) | {"_init", "_fini"}, sorted(exported - set(declared()))


def test_invalid_arguments_are_reported(vl):
    with pytest.raises(vl.VljError) as e:
        vl.lattice(0, 1.0, 1.0, 1)
    assert e.value.status == "INVALID_ARG"
    with pytest.raises(vl.VljError):
        vl.lattice_box(10, [1.0, -1.0, 1.0], 1.0, 1)


def test_profile_phases_of_two_slabs_across_the_boundary(vl):
    # lennard_jones.rs:1468-1497
    density = [0.7 if (b < 10 or 50 <= b < 60 or 25 <= b < 40) else 0.02 for b in range(60)]
    slabs = [vl.Slab(b + 0.5, rho, [0.0] * 3, [0.0] * 3, 0.0) for b, rho in enumerate(density)]
    p = vl.Profile(1, [1.0, 1.0, 60.0], slabs)
    assert sorted(p.interfaces(0.36)) == [10.0, 25.0, 40.0, 50.0]
    phases = p.phases(0.36, 4.0)
    count = lambda q: sum(1 for x in phases if x == q)
    assert count(vl.Phase.LIQUID) == 6 + 6 + 7
    assert abs(p.mean_in(density, phases, vl.Phase.LIQUID) - 0.7) < 1e-12
    assert abs(p.mean_in(density, phases, vl.Phase.VAPOUR) - 0.02) < 1e-12
    assert count(vl.Phase.INTERFACE) == 4 * 4
    flat = vl.Profile(1, [1.0, 1.0, 8.0], [vl.Slab(b + 0.5, 0.3, [0.0] * 3, [0.0] * 3, 0.0)
                                           for b in range(8)])
    assert all(q == vl.Phase.BETWEEN for q in flat.phases(0.36, 4.0))


def test_create_without_device_fails_loudly(vl):
    if vl.device_count() > 0:
        pytest.skip("a device is present")
    p = vl.lattice(1000, 11.0, 1.0, 3)
    with pytest.raises(vl.VljError) as e:
        vl.LennardJones(p, vl.Settings([11.0] * 3))
    assert e.value.status == "NO_DEVICE"


def header_arities():
    """Parameter count of every function the header declares."""
    text = open(os.path.join(ROOT, "include", "virial_lj.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"VLJ_API\s+[\w\s\*]+?\b(vlj_\w+)\s*\(([^)]*)\)", text):
        args = " ".join(m.group(2).split())
        out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_python_signatures_match_the_header():
    # the ctypes table passes exactly the arguments each C function takes
    import sys
    sys.path.insert(0, os.path.join(ROOT, "virial-engine_b200"))
    from virial_lj import _ffi
    arity = header_arities()
    assert set(_ffi.SIGNATURES) <= set(arity), sorted(set(_ffi.SIGNATURES) - set(arity))
    wrong = {n: (len(t), arity[n]) for n, t in _ffi.SIGNATURES.items() if len(t) != arity[n]}
    assert not wrong, wrong
