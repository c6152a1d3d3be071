"""The C++ host layer (n-body_b200/host/nbody_b200.hpp) through its command-line runner, on a GPU.

The C++ Solver classes drive the same C ABI as the Python binding, so a scenario stepped by
nbody_cli must end bit-identical to the same steps through the binding, with the same
interaction counts.
"""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import REPO

pytestmark = pytest.mark.gpu

CLI = os.path.join(REPO, "n-body_b200", "lib", "nbody_cli")


def run(*args):
    r = subprocess.run([CLI, *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r


@pytest.mark.parametrize("solver_id,cls,theta,leaf,steps", [
    ("linear-bvh", "LinearBVHSolver", 0.5, 16, 3),
    ("linear-bvh-4p", "QuadrupoleLinearBVHSolver", 0.5, 16, 4),
    ("naive", "NaiveSolver", 0.5, 16, 2),
    ("implicit-linear-bvh-fmm-8p", "OctupoleImplicitLinearBVHFMMSolver", 0.4, 64, 2),
])
def test_cli_matches_binding(tmp_path, nb, solver_id, cls, theta, leaf, steps):
    pm, vel = nb.scenarios.plummer(6000, seed=17)
    src = tmp_path / "in.json"
    nb.scenarios.write_json(str(src), pm, vel, G=1.5)
    out = tmp_path / "out.json"
    r = run("-s", solver_id, "-i", str(steps), "-t", "0.001", "--theta", str(theta), "--max-leaf-size", str(leaf),
            "--epsilon", "0.0001", "-o", str(out), "--counts", str(src))
    counts = json.loads(r.stdout.strip().splitlines()[-1])
    assert counts["solver"] == solver_id
    p_cli, v_cli, a_cli, G = nb.scenarios.read_json(str(out))
    assert G == np.float32(1.5)
    with getattr(nb, cls)(bodies=pm, velocities=vel, rule=nb.Gravity(1.5, 1e-4), theta=theta, max_leaf_size=leaf,
                          time_step=1e-3) as s:
        s.step(steps)
        p_ref, v_ref = s.bodies()
        a_ref = s.accelerations()
        c_ref = s.counts()
    assert np.array_equal(p_cli, p_ref)
    assert np.array_equal(v_cli[:, :3], v_ref[:, :3])
    assert np.array_equal(a_cli[:, :3], a_ref[:, :3])
    for k in ("particle_particle", "particle_node", "node_particle", "node_node"):
        assert counts[k] == c_ref[k], k


@pytest.mark.parametrize("solver_id,theta,leaf", [
    ("linear-bvh-4p", 0.5, 16),
    ("implicit-linear-bvh-fmm-8p", 0.4, 64),
])
def test_cli_checkpoint_resume_is_exact(tmp_path, nb, solver_id, theta, leaf):
    """A checkpoint is a scenario: resuming from the step-2 checkpoint for 3 more steps ends
    bit-identical to 5 uninterrupted steps (each step recomputes the accelerations from the
    positions, and %.9g round-trips every float)."""
    pm, vel = nb.scenarios.plummer(5000, seed=23)
    src = tmp_path / "in.json"
    nb.scenarios.write_json(str(src), pm, vel, G=0.75)
    common = ["-s", solver_id, "-t", "0.001", "--theta", str(theta), "--max-leaf-size", str(leaf),
              "--epsilon", "0.0002"]
    straight = tmp_path / "straight.json"
    run(*common, "-i", "5", "-o", str(straight), str(src))
    prefix = str(tmp_path / "ckpt")
    chunked = tmp_path / "chunked.json"
    run(*common, "-i", "5", "--checkpoint-every", "2", "--checkpoint-prefix", prefix, "-o", str(chunked), str(src))
    assert sorted(os.listdir(tmp_path)) == sorted(["in.json", "straight.json", "chunked.json", "ckpt.2.json",
                                                   "ckpt.4.json", "ckpt.5.json"])
    resumed = tmp_path / "resumed.json"
    run(*common, "-i", "3", "-o", str(resumed), prefix + ".2.json")
    p0, v0, _, G0 = nb.scenarios.read_json(str(straight))
    for path in (chunked, resumed, prefix + ".5.json"):
        p, v, _, G = nb.scenarios.read_json(str(path))
        assert G == G0 == np.float32(0.75)
        assert np.array_equal(p, p0), path
        assert np.array_equal(v[:, :3], v0[:, :3]), path


def test_cli_verbose_steps_on_background_thread(tmp_path, nb):
    """--verbose steps one at a time through Solver::stepAsync (the reference's slot_step) and
    prints each step's compute time; the result equals stepping in one call, bit for bit."""
    pm, vel = nb.scenarios.plummer(4000, seed=29)
    src = tmp_path / "in.json"
    nb.scenarios.write_json(str(src), pm, vel)
    common = ["-s", "linear-bvh-4p", "-i", "4", "-t", "0.001", "--epsilon", "0.0001"]
    plain, verbose = tmp_path / "plain.json", tmp_path / "verbose.json"
    run(*common, "-o", str(plain), str(src))
    r = run(*common, "--verbose", "-o", str(verbose), str(src))
    lines = [l for l in r.stderr.splitlines() if l.startswith("step ")]
    assert [l.split(":")[0] for l in lines] == ["step 1", "step 2", "step 3", "step 4"]
    assert all(float(l.split(":")[1].split()[0]) > 0 for l in lines)
    p0, v0, _, _ = nb.scenarios.read_json(str(plain))
    p1, v1, _, _ = nb.scenarios.read_json(str(verbose))
    assert np.array_equal(p0, p1)
    assert np.array_equal(v0[:, :3], v1[:, :3])


MULTI_PROGRAM = r"""
#include "nbody_b200.hpp"
#include "scenario.hpp"
#include <cstdio>
#include <fstream>
using namespace nbody_b200;
static void configure(MultiSolver &ms) {
    ms.get().setTheta(0.5f);
    ms.get().setMaxLeafSize(16);
    ms.get().setTimeStep(0.001f);
}
int main(int argc, char **argv) {
    Scenario sc = load_scenario(argv[1]);
    Gravity rule(1.0f, 1e-4f);
    MultiSolver ms(sc.simulation, rule, "linear-bvh-4p");
    configure(ms);
    ms.step(3);
    ms.select("naive");
    configure(ms);
    ms.step(1);
    ms.select(1);  // linear-bvh-4p again: it resumes from the simulation's current bodies
    configure(ms);
    ms.step(1);
    std::ofstream(argv[2]) << scenario_to_json(sc.simulation, nullptr);
    std::printf("%s\n", ms.id().c_str());
}
"""


def test_multisolver_switches_between_solvers(tmp_path, nb):
    """MultiSolver::select switches algorithms on one simulation; each step equals the same step
    through that solver class alone, bit for bit."""
    src = tmp_path / "multi.cpp"
    src.write_text(MULTI_PROGRAM)
    exe = tmp_path / "multi"
    lib = os.path.join(REPO, "n-body_b200", "lib")
    host = os.path.join(REPO, "n-body_b200", "host")
    subprocess.run(["g++", "-std=c++17", "-I", host, "-o", str(exe), str(src), "-L", lib, "-lnbody_b200",
                    "-Wl,-rpath," + lib], check=True)
    pm, vel = nb.scenarios.plummer(3000, seed=41)
    scen = tmp_path / "in.json"
    nb.scenarios.write_json(str(scen), pm, vel)
    out = tmp_path / "out.json"
    r = subprocess.run([str(exe), str(scen), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "linear-bvh-4p"
    p_cpp, v_cpp, _, _ = nb.scenarios.read_json(str(out))
    rule = nb.Gravity(1.0, 1e-4)
    kw = dict(rule=rule, theta=0.5, max_leaf_size=16, time_step=1e-3)
    with nb.QuadrupoleLinearBVHSolver(bodies=pm, velocities=vel, **kw) as s:
        s.step(3)
        p, v = s.bodies()
    with nb.NaiveSolver(bodies=p, velocities=v, **kw) as s:
        s.step(1)
        p, v = s.bodies()
    with nb.QuadrupoleLinearBVHSolver(bodies=p, velocities=v, **kw) as s:
        s.step(1)
        p, v = s.bodies()
    assert np.array_equal(p_cpp, p)
    assert np.array_equal(v_cpp[:, :3], v[:, :3])
