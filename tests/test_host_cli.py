"""The C++ host layer's scenario I/O and command line, without a GPU.

nbody_cli reads the reference's JSON scenario schema (Simulation.cpp:154-228) and tipsy files
(Simulation.cpp:273-395) and writes JSON; with --iterations 0 it converts without touching the
device. With iterations it must fail loudly when no sm_100 device is present (no CPU fallback).
"""
import json
import os
import struct
import subprocess

import numpy as np
import pytest

from conftest import REPO

CLI = os.path.join(REPO, "n-body_b200", "lib", "nbody_cli")


def run(*args):
    return subprocess.run([CLI, *args], capture_output=True, text=True, timeout=120)


@pytest.fixture(scope="module", autouse=True)
def built():
    if not os.path.exists(CLI):
        subprocess.run(["make", "-C", os.path.join(REPO, "n-body_b200"), "-s"], check=True)
    assert os.path.exists(CLI)


def test_json_round_trip(tmp_path, nb):
    pm, vel = nb.scenarios.plummer(257, seed=3)
    src = tmp_path / "in.json"
    # extra keys of the reference's files (colour, sphere) are ignored
    nb.scenarios.write_json(str(src), pm, vel, G=2.5)
    root = json.load(open(src))
    root["particles"][0]["color"] = {"r": 0.8, "g": 0.0, "b": 0.0}
    root["particles"][0]["sphere"] = {"radius": 1.0}
    json.dump(root, open(src, "w"))
    out = tmp_path / "out.json"
    r = run("-i", "0", "-o", str(out), str(src))
    assert r.returncode == 0, r.stderr
    pm2, vel2, acc2, G = nb.scenarios.read_json(str(out))
    assert np.array_equal(pm2, pm)
    assert np.array_equal(vel2[:, :3], vel[:, :3])
    assert not acc2.any()
    assert G == np.float32(2.5)


def test_json_missing_components_default_to_zero(tmp_path, nb):
    src = tmp_path / "in.json"
    src.write_text(json.dumps({"particles": [{"position": {"x": 1, "y": 2, "z": 3}, "mass": 0.5},
                                             {"velocity": {"x": 0.5, "y": 0, "z": 0}}]}))
    out = tmp_path / "out.json"
    assert run("-i", "0", "-o", str(out), str(src)).returncode == 0
    pm, vel, acc, G = nb.scenarios.read_json(str(out))
    assert G is None
    assert pm.tolist() == [[1, 2, 3, 0.5], [0, 0, 0, 0]]
    assert vel[:, :3].tolist() == [[0, 0, 0], [0.5, 0, 0]]


def test_json_errors_fail(tmp_path):
    bad = tmp_path / "bad.json"
    bad.write_text('{"particles": [ {"position": {"x": 1, "y": 2}} ]}')
    r = run("-i", "0", "-o", str(tmp_path / "o.json"), str(bad))
    assert r.returncode == 1 and "lacks z" in r.stderr
    bad.write_text('{"particles": [ }')
    assert run("-i", "0", str(bad)).returncode == 1
    bad.write_text('{"bodies": []}')
    assert run("-i", "0", str(bad)).returncode == 1


def write_tipsy(path, gas, dark, stars, big_endian=False, pad=False, time=0.0):
    """Tipsy file: header (double time; uint32 n, ndim, ngas, ndark, nstar) [+ 4-byte pad], then
    gas (12 floats), dark (9 floats), stars (11 floats) per particle."""
    e = ">" if big_endian else "<"
    n = len(gas) + len(dark) + len(stars)
    with open(path, "wb") as f:
        f.write(struct.pack(e + "dIIIII", time, n, 3, len(gas), len(dark), len(stars)))
        if pad:
            f.write(b"\0\0\0\0")
        for rows, width in ((gas, 12), (dark, 9), (stars, 11)):
            for row in rows:
                assert len(row) == width
                f.write(struct.pack(e + "f" * width, *row))


def tipsy_rows(rng, count, width):
    return rng.normal(size=(count, width)).astype(np.float32).tolist()


@pytest.mark.parametrize("big_endian,pad", [(False, False), (True, False), (False, True), (True, True)])
def test_tipsy_gas_only(tmp_path, nb, big_endian, pad):
    rng = np.random.default_rng(1)
    gas = tipsy_rows(rng, 40, 12)
    dark = tipsy_rows(rng, 7, 9)
    path = tmp_path / "g.bin"
    write_tipsy(path, gas, dark, [], big_endian, pad)
    out = tmp_path / "out.json"
    r = run("-i", "0", "-o", str(out), str(path))
    assert r.returncode == 0, r.stderr
    pm, vel, _, _ = nb.scenarios.read_json(str(out))
    g = np.array(gas, np.float32)
    # without stars, gas is read (mass, position, velocity) and dark matter is skipped
    assert np.array_equal(pm[:, 3], g[:, 0])
    assert np.array_equal(pm[:, :3], g[:, 1:4])
    assert np.array_equal(vel[:, :3], g[:, 4:7])


def test_tipsy_stars_skip_gas_and_dark(tmp_path, nb):
    rng = np.random.default_rng(2)
    gas, dark, stars = tipsy_rows(rng, 5, 12), tipsy_rows(rng, 6, 9), tipsy_rows(rng, 9, 11)
    path = tmp_path / "s.bin"
    write_tipsy(path, gas, dark, stars, big_endian=True, pad=True)
    out = tmp_path / "out.json"
    assert run("-i", "0", "-o", str(out), str(path)).returncode == 0
    pm, vel, _, _ = nb.scenarios.read_json(str(out))
    s = np.array(stars, np.float32)
    assert len(pm) == 9
    assert np.array_equal(pm[:, 3], s[:, 0])
    assert np.array_equal(pm[:, :3], s[:, 1:4])
    assert np.array_equal(vel[:, :3], s[:, 4:7])


def test_tipsy_size_mismatch_fails(tmp_path):
    rng = np.random.default_rng(3)
    path = tmp_path / "t.bin"
    write_tipsy(path, tipsy_rows(rng, 3, 12), [], [])
    with open(path, "ab") as f:
        f.write(b"\0" * 7)
    r = run("-i", "0", str(path))
    assert r.returncode == 1 and "does not match" in r.stderr


def test_cli_without_gpu_fails_loudly(tmp_path, nb):
    """No CPU fallback: stepping needs the device and fails with a message when there is none."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    pm, vel = nb.scenarios.uniform_ball(64, seed=1)
    src = tmp_path / "in.json"
    nb.scenarios.write_json(str(src), pm, vel)
    r = run("-s", "linear-bvh-4p", "-i", "2", "-o", str(tmp_path / "o.json"), str(src))
    assert r.returncode == 1 and "nb_create failed" in r.stderr
    assert not (tmp_path / "o.json").exists()


def test_cli_rejects_bad_arguments(tmp_path, nb):
    pm, vel = nb.scenarios.uniform_ball(8, seed=1)
    src = tmp_path / "in.json"
    nb.scenarios.write_json(str(src), pm, vel)
    assert run().returncode == 2
    assert run("--bogus", str(src)).returncode == 2
    r = run("-s", "barnes-hut-octree", "-i", "1", str(src))
    assert r.returncode == 1 and "unknown solver id" in r.stderr
    # a checkpoint interval needs a prefix and must not be negative
    assert run("-i", "2", "--checkpoint-every", "1", str(src)).returncode == 2
    assert run("-i", "2", "--checkpoint-every", "-1", "--checkpoint-prefix", str(tmp_path / "c"), str(src)).returncode == 2


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", ["threebody.json", "test.json"])
def test_reads_reference_scenario_files(tmp_path, nb, name):
    """The reference's own scenario files (scenarios/*.json), kept as fixtures in tests/golden."""
    src = os.path.join(GOLDEN, name)
    out = tmp_path / "out.json"
    r = run("-i", "0", "-o", str(out), src)
    assert r.returncode == 0, r.stderr
    root = json.load(open(src))
    pm, vel, _, G = nb.scenarios.read_json(str(out))
    assert len(pm) == len(root["particles"])
    for i, p in enumerate(root["particles"]):
        if "position" in p:
            assert pm[i, :3].tolist() == [np.float32(p["position"][c]) for c in "xyz"]
        if "velocity" in p:
            assert vel[i, :3].tolist() == [np.float32(p["velocity"][c]) for c in "xyz"]
        assert pm[i, 3] == np.float32(p.get("mass", 0.0))
    assert (G is None) == ("G" not in root)


HOST_PROGRAM = r"""
#include "nbody_b200.hpp"
#include <cstdio>
int main() {
    nbody_b200::Simulation s;
    s.newParticle({1, 2, 3}, {0, 0, 0}, 2.f);
    s.newParticle({-1, 0, 5}, {0, 0, 0}, 1.f);
    s.newParticle({4, -2, 1}, {1, 0, 0}, 1.f);
    const auto c = s.centerOfMass(), a = s.averagePosition();
    const auto b = s.boundingBox();
    std::printf("%.9g %.9g %.9g\n%.9g %.9g %.9g\n", c.x, c.y, c.z, a.x, a.y, a.z);
    std::printf("%.9g %.9g %.9g %.9g %.9g %.9g\n", b.min.x, b.min.y, b.min.z, b.max.x, b.max.y, b.max.z);
    std::printf("%.9g %zu %d %d\n", s.totalMass(), s.interactionCount(), (int) b.contains({0, 0, 3}),
                (int) b.contains(b.max));
    s.removeParticle(0);
    std::printf("%zu %.9g %.9g\n", s.particleCount(), s.position[0].x, s.mass[1]);
    nbody_b200::BoundingBox empty;
    std::printf("%d\n", (int) (empty.min.x > empty.max.x));
}
"""


def test_simulation_helpers(tmp_path):
    """Simulation's host-side summaries (averagePosition, totalMass, centerOfMass, boundingBox,
    interactionCount, removeParticle) as the reference defines them (Simulation.cpp:73-132)."""
    src = tmp_path / "sim.cpp"
    src.write_text(HOST_PROGRAM)
    exe = tmp_path / "sim"
    subprocess.run(["g++", "-std=c++20", "-I", os.path.join(REPO, "n-body_b200", "host"), "-o", str(exe), str(src)],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    f32 = np.float32
    pos = np.array([[1, 2, 3], [-1, 0, 5], [4, -2, 1]], f32)
    m = np.array([2, 1, 1], f32)
    com = ((pos[0] * m[0] + pos[1] * m[1]) + pos[2] * m[2]) / ((m[0] + m[1]) + m[2])
    avg = ((pos[0] + pos[1]) + pos[2]) / f32(3)
    assert [f32(v) for v in out[0].split()] == list(com)
    assert [f32(v) for v in out[1].split()] == list(avg)
    assert [float(v) for v in out[2].split()] == [-1, -2, 1, 4, 2, 5]
    assert out[3].split() == ["4", "9", "1", "0"]  # the box is half-open: its max corner is outside
    assert out[4].split() == ["2", "-1", "1"]
    assert out[5] == "1"


MULTI_PROGRAM = r"""
#include "nbody_b200.hpp"
#include <cstdio>
#include <cstring>
int main(int argc, char **argv) {
    nbody_b200::Simulation sim;
    sim.newParticle({0, 0, 0}, {0, 0, 0}, 1.f);
    sim.newParticle({1, 0, 0}, {0, 0, 0}, 1.f);
    nbody_b200::Gravity rule;
    try {
        nbody_b200::MultiSolver ms(sim, rule, argv[1]);
        std::printf("selected %s\n", ms.id().c_str());
    } catch (const nbody_b200::Error &e) {
        std::printf("error %s\n", e.what());
    }
}
"""


def build_multi(tmp_path):
    src = tmp_path / "multi.cpp"
    src.write_text(MULTI_PROGRAM)
    exe = tmp_path / "multi"
    lib = os.path.join(REPO, "n-body_b200", "lib")
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(REPO, "n-body_b200", "host"), "-o", str(exe), str(src),
                    "-L", lib, "-lnbody_b200", "-Wl,-rpath," + lib], check=True)
    return exe


def test_multisolver_rejects_unknown_ids(tmp_path):
    """MultiSolver::select with an id the device path does not implement fails before any device
    work (the reference logs "Unrecognized solver id", MultiSolver.h:79-87)."""
    exe = build_multi(tmp_path)
    out = subprocess.run([str(exe), "barnes-hut-octree"], capture_output=True, text=True, check=True).stdout
    assert out.strip() == "error unknown solver id: barnes-hut-octree"


def test_multisolver_without_gpu_fails_loudly(tmp_path):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    exe = build_multi(tmp_path)
    out = subprocess.run([str(exe), "linear-bvh-4p"], capture_output=True, text=True, check=True).stdout
    assert out.startswith("error nb_create failed")
