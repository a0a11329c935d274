/*
 * main() of HPM-MVS (main.cpp:636-677) on the B200 path: pass set A
 * (ProcessProblem with the planar prior) for every problem of pair.txt, two
 * geometric-consistency iterations over every problem, then the fusion
 * into HPM/HPM_model.ply (RunFusion, main.cpp:502-633).
 *
 *   hpm_mvs dense_folder [--seed S] [--levels K] [--device D] [--no-prior]
 *                        [--geom-iterations G] [--no-fusion] [--per-problem]
 *
 * By default the passes run as one scene (RunScene: maps in device memory
 * between passes, pass set A on two host threads, files written at the
 * end); --per-problem runs ProcessProblem problem by problem as the
 * reference does, reading and writing the .dmb files between passes.
 * Problem p of pass set A uses seed S + p; problem p of geometric iteration
 * g uses S + 1000003 (g + 1) + p, in both forms, so both write the same
 * files.
 */
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "hpm_host.h"

int main(int argc, char **argv)
{
    if (argc < 2 || !strcmp(argv[1], "-h") || !strcmp(argv[1], "--help")) {
        std::cout << "USAGE: hpm_mvs dense_folder [--seed S] [--levels K] [--device D] [--no-prior] "
                     "[--geom-iterations G] [--no-fusion] [--per-problem]"
                  << std::endl;
        return argc < 2 ? -1 : 0;
    }
    const std::string dense_folder = argv[1];
    uint64_t seed = 0;
    int levels = -1, device = 0, geom_iterations = 2;
    bool planar_prior = true, fusion = true, per_problem = false;
    for (int i = 2; i < argc; ++i) {
        const std::string a = argv[i];
        auto next = [&](const char *name) -> const char * {
            if (i + 1 >= argc) {
                std::cerr << name << " needs a value" << std::endl;
                std::exit(2);
            }
            return argv[++i];
        };
        if (a == "--seed")
            seed = std::strtoull(next("--seed"), nullptr, 10);
        else if (a == "--levels")
            levels = std::atoi(next("--levels"));
        else if (a == "--device")
            device = std::atoi(next("--device"));
        else if (a == "--geom-iterations")
            geom_iterations = std::atoi(next("--geom-iterations"));
        else if (a == "--no-prior")
            planar_prior = false;
        else if (a == "--no-fusion")
            fusion = false;
        else if (a == "--per-problem")
            per_problem = true;
        else {
            std::cerr << "unknown option " << a << std::endl;
            return 2;
        }
    }
    try {
        std::vector<hpm_host::Problem> problems;
        hpm_host::GenerateSampleList(dense_folder, problems);
        std::cout << "There are " << problems.size() << " problems needed to be processed!" << std::endl;
        if (!per_problem) {
            hpm_host::RunScene(dense_folder, problems, planar_prior, geom_iterations, seed, levels, device);
        } else {
            for (size_t p = 0; p < problems.size(); ++p)
                hpm_host::ProcessProblem(dense_folder, problems[p], false, planar_prior, false, seed + p, levels,
                                         device);
            for (int g = 0; g < geom_iterations; ++g)
                for (size_t p = 0; p < problems.size(); ++p)
                    hpm_host::ProcessProblem(dense_folder, problems[p], true, false, g > 0,
                                             seed + 1000003ull * (g + 1) + p, levels, device);
        }
        if (fusion) {
            const long long n = hpm_host::RunFusion(dense_folder, problems, geom_iterations > 0, device);
            std::cout << "Fused " << n << " points into " << dense_folder << "/HPM/HPM_model.ply" << std::endl;
        }
    } catch (const hpm_host::Error &e) {
        std::cerr << "hpm_mvs: " << e.what() << " (status " << e.code << ")" << std::endl;
        return 1;
    }
    return 0;
}
