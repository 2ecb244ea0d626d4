"""The C++ mirror of the reference API (include/virial_lj.hpp) compiles against
the C ABI, links the library, and passes the reference's tests restated in C++
(tests/cpp/test_lj.cpp): host-only ones here, all of them on a GPU."""

import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build(vl, out_dir):
    lib_dir = os.path.dirname(vl.library_path())
    exe = os.path.join(out_dir, "test_lj")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror",
           "-I" + os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "test_lj.cpp"),
           "-L" + lib_dir, "-lvirial_lj", "-Wl,-rpath," + lib_dir, "-o", exe]
    done = subprocess.run(cmd, capture_output=True, text=True)
    assert done.returncode == 0, done.stderr
    return exe


def run(exe, mode, timeout):
    done = subprocess.run([exe, mode], capture_output=True, text=True, timeout=timeout)
    print(done.stdout)
    assert done.returncode == 0, done.stdout + done.stderr
    assert done.stdout.strip().endswith("0 failed")
    return done.stdout


def test_cpp_mirror_host_entry_points(vl, tmp_path):
    out = run(build(vl, str(tmp_path)), "host", 120)
    assert "ok   phases_of_two_slabs_across_the_boundary" in out


@pytest.mark.gpu
def test_cpp_mirror_reference_tests(gpu, tmp_path):
    out = run(build(gpu, str(tmp_path)), "gpu", 600)
    for name in ["cell_grid_finds_every_pair", "rectangular_box_matches_all_pairs",
                 "profiles_add_up_to_the_whole_box", "thermostatted_reruns_are_bit_identical",
                 "heat_exchange_moves_energy_and_keeps_momentum",
                 "measurements_arrive_in_order", "panics_become_errors"]:
        assert "ok   " + name in out
