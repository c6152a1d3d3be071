// Command-line runner of the device force path, with the reference CLI's options
// (src/Application/Application.cpp:22-131):
//
//   nbody_cli [-s|--solver ID] [-i|--iterations N] [-t|--timestep DT] [-G|--gravity G]
//             [-o|--output-file PATH] [--theta T] [--max-leaf-size L] [--epsilon E]
//             [--device D] [--counts] [--checkpoint-every K --checkpoint-prefix P] [--verbose]
//             SCENARIO
//
// SCENARIO is a JSON scenario (the reference's schema; a top-level "G" sets the constant, as
// Application::on_open does) or a tipsy file. The solver ids are the reference's Solver::id()
// strings. With --iterations 0 nothing runs on the device and the scenario is only converted
// (JSON out), so I/O needs no GPU. The result is written as a JSON scenario; --counts prints the
// last force pass's interaction counts as one JSON line on stdout. --checkpoint-every K writes the
// state every K steps to P.<step>.json (the same schema, so a checkpoint resumes as a scenario).
// --verbose runs one step at a time on the solver's background thread (stepAsync, the reference's
// slot_step) and prints each step's compute time, as the reference's computeTime signal reports it.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>

#include "nbody_b200.hpp"
#include "scenario.hpp"

using namespace nbody_b200;

namespace {

void usage() {
    std::fprintf(stderr,
                 "usage: nbody_cli [-s ID] [-i N] [-t DT] [-G G] [-o OUT.json] [--theta T] [--max-leaf-size L]\n"
                 "                 [--epsilon E] [--device D] [--counts] [--checkpoint-every K --checkpoint-prefix P]\n"
                 "                 [--verbose]\n"
                 "                 SCENARIO(.json|tipsy)\n"
                 "solvers:");
    for (auto &id: solverIds()) std::fprintf(stderr, " %s", id.c_str());
    std::fprintf(stderr, "\n");
}

struct Options {
    std::string solver = "linear-bvh-4p", input, output, checkpoint_prefix;
    int iterations = 0, device = 0, leaf = -1, checkpoint_every = 0;
    bool has_dt = false, has_G = false, has_theta = false, has_eps = false, counts = false, verbose = false;
    double dt = 0.0, G = 1.0, theta = 0.0, eps = 0.0;
};

bool parse(int argc, char **argv, Options &o) {
    for (int k = 1; k < argc; ++k) {
        const std::string a = argv[k];
        auto next = [&]() -> const char * {
            if (k + 1 >= argc) {
                std::fprintf(stderr, "missing value for %s\n", a.c_str());
                std::exit(2);
            }
            return argv[++k];
        };
        if (a == "-s" || a == "--solver") o.solver = next();
        else if (a == "-i" || a == "--iterations") o.iterations = std::atoi(next());
        else if (a == "-t" || a == "--timestep") { o.dt = std::atof(next()); o.has_dt = true; }
        else if (a == "-G" || a == "--gravity") { o.G = std::atof(next()); o.has_G = true; }
        else if (a == "-o" || a == "--output-file") o.output = next();
        else if (a == "--theta") { o.theta = std::atof(next()); o.has_theta = true; }
        else if (a == "--max-leaf-size") o.leaf = std::atoi(next());
        else if (a == "--epsilon") { o.eps = std::atof(next()); o.has_eps = true; }
        else if (a == "--device") o.device = std::atoi(next());
        else if (a == "--counts") o.counts = true;
        else if (a == "--verbose") o.verbose = true;
        else if (a == "--checkpoint-every") o.checkpoint_every = std::atoi(next());
        else if (a == "--checkpoint-prefix") o.checkpoint_prefix = next();
        else if (a == "-h" || a == "--help") return false;
        else if (!a.empty() && a[0] == '-') {
            std::fprintf(stderr, "unknown option %s\n", a.c_str());
            return false;
        } else o.input = a;
    }
    if (o.checkpoint_every < 0 || (o.checkpoint_every > 0 && o.checkpoint_prefix.empty())) return false;
    return !o.input.empty() && o.iterations >= 0;
}

}  // namespace

int main(int argc, char **argv) {
    Options o;
    if (!parse(argc, argv, o)) {
        usage();
        return 2;
    }
    try {
        Scenario sc = load_scenario(o.input);
        Gravity rule;
        if (sc.hasG) rule.g() = sc.G;
        if (o.has_G) rule.g() = (float) o.G;
        if (o.has_eps) rule.epsilon() = (float) o.eps;
        Simulation &sim = sc.simulation;
        InteractionCounts counts;
        std::string solver_id;
        if (o.iterations > 0) {
            auto solver = makeSolver(o.solver, sim, rule);
            if (o.has_theta) solver->setTheta((float) o.theta);
            if (o.leaf > 0) solver->setMaxLeafSize(o.leaf);
            if (o.has_dt) solver->setTimeStep((float) o.dt);
            const float G = rule.g();
            int done = 0;
            if (o.verbose)
                solver->onComputeTime([&](std::chrono::duration<double> d) {
                    std::fprintf(stderr, "step %d: %.6f s\n", done + 1, d.count());
                });
            // device-resident steps between checkpoints; each checkpoint copies the state out once
            const int chunk = o.verbose ? 1 : (o.checkpoint_every > 0 ? o.checkpoint_every : o.iterations);
            while (done < o.iterations) {
                const int k = std::min(chunk, o.iterations - done);
                if (o.verbose) {
                    solver->stepAsync();
                    solver->wait();
                } else {
                    solver->step(k);
                }
                done += k;
                if (o.checkpoint_every > 0 && (done % o.checkpoint_every == 0 || done == o.iterations)) {
                    const std::string path = o.checkpoint_prefix + "." + std::to_string(done) + ".json";
                    std::ofstream out(path);
                    out << scenario_to_json(sim, sc.hasG || o.has_G ? &G : nullptr);
                    if (!out.good()) throw Error(NB_ERR_INVALID_ARGUMENT, "cannot write " + path);
                }
            }
            counts = solver->counts();
            solver_id = solver->id();
        }
        if (!o.output.empty()) {
            std::ofstream out(o.output);
            const float G = rule.g();
            out << scenario_to_json(sim, sc.hasG || o.has_G ? &G : nullptr);
            if (!out.good()) throw Error(NB_ERR_INVALID_ARGUMENT, "cannot write " + o.output);
        }
        if (o.counts)
            std::printf("{\"solver\": \"%s\", \"particles\": %zu, \"iterations\": %d, \"particle_particle\": %llu, "
                        "\"particle_node\": %llu, \"node_particle\": %llu, \"node_node\": %llu}\n",
                        solver_id.c_str(), sim.particleCount(), o.iterations,
                        (unsigned long long) counts.particleParticle, (unsigned long long) counts.particleNode,
                        (unsigned long long) counts.nodeParticle, (unsigned long long) counts.nodeNode);
    } catch (const Error &e) {
        std::fprintf(stderr, "nbody_cli: %s (status %d)\n", e.what(), e.status());
        return 1;
    }
    return 0;
}
