/*
 * main() of HPM-MVS (main.cpp:636-677) on the B200 path: pass set A
 * (ProcessProblem with the planar prior) for every problem of pair.txt, two
 * geometric-consistency iterations over every problem, then the fusion
 * into HPM/HPM_model.ply (RunFusion, main.cpp:502-633).
 *
 *   hpm_mvs dense_folder [--seed S] [--levels K] [--device D] [--no-prior]
 *                        [--geom-iterations G] [--no-fusion] [--per-problem]
 *                        [--resume] [--stop-after N] [--no-reference-compat] [--log PATH]
 *
 * By default the passes run as one scene (RunScene: maps in device memory
 * between passes, pass set A on two host threads, files written at the
 * end); --per-problem runs ProcessProblem problem by problem as the
 * reference does, reading and writing the .dmb files between passes.
 * Problem p of pass set A uses seed S + p; problem p of geometric iteration
 * g uses S + 1000003 (g + 1) + p, in both forms, so both write the same
 * files.
 *
 * Every finished step is logged in HPM/progress.txt (hpm_host::Progress).
 * --stop-after N ends the run, with status 0, once N steps of this run have
 * finished (a problem of pass set A or of a geometric iteration, the scene
 * of the scene form, the fusion); --resume skips the steps the log holds, so
 * a scene can be computed in several runs.  Both forms resume to the files
 * one uninterrupted run writes.
 *
 * --log PATH appends one JSON line per finished step to PATH: the step, its
 * wall time, and the depth pixels it wrote with their rate (for the fusion,
 * the points).
 *
 * The reference's behaviour is kept throughout by default (its quirks
 * included); --no-reference-compat fixes the quirks listed at HpmParams in
 * hpm_b200.h.
 *
 * --acmm runs the reference's other product instead, the ACMM+NESP
 * variant's main() (ACMM+NESP/windows/main.cpp:299-384): coarse-to-fine
 * over an image pyramid (RunSceneAcmm), files under ACMM_NESP/2333_%08d/,
 * fused into ACMM_NESP/ACMM_NESP_model.ply.
 */
#include <chrono>
#include <cstdlib>
#include <fstream>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "hpm_host.h"

int main(int argc, char **argv)
{
    if (argc < 2 || !strcmp(argv[1], "-h") || !strcmp(argv[1], "--help")) {
        std::cout << "USAGE: hpm_mvs dense_folder [--seed S] [--levels K] [--device D] [--no-prior] "
                     "[--geom-iterations G] [--no-fusion] [--per-problem] [--resume] [--stop-after N] "
                     "[--no-reference-compat] [--log PATH] [--acmm]"
                  << std::endl;
        return argc < 2 ? -1 : 0;
    }
    const std::string dense_folder = argv[1];
    uint64_t seed = 0;
    int levels = -1, device = 0, geom_iterations = 2;
    bool planar_prior = true, fusion = true, per_problem = false, resume = false, compat = true, acmm = false;
    long long stop_after = -1;
    std::string log_path;
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
        else if (a == "--resume")
            resume = true;
        else if (a == "--no-reference-compat")
            compat = false;
        else if (a == "--acmm")
            acmm = true;
        else if (a == "--log")
            log_path = next("--log");
        else if (a == "--stop-after")
            stop_after = std::atoll(next("--stop-after"));
        else {
            std::cerr << "unknown option " << a << std::endl;
            return 2;
        }
    }
    try {
        std::vector<hpm_host::Problem> problems;
        hpm_host::GenerateSampleList(dense_folder, problems);
        std::cout << "There are " << problems.size() << " problems needed to be processed!" << std::endl;
        std::ostringstream settings;
        settings << "seed=" << seed << " levels=" << levels << " prior=" << planar_prior
                 << " geom_iterations=" << geom_iterations << " form="
                 << (acmm ? "acmm" : (per_problem ? "per-problem" : "scene"))
                 << (compat ? "" : " fix_quirks=1");
        hpm_host::Progress progress(dense_folder, settings.str(), resume);
        long long steps = 0;
        /* runs one step unless the log holds it; false once --stop-after is
         * reached.  work() returns the depth pixels it wrote (the fusion: its
         * points, as a negative number) */
        auto step = [&](const std::string &name, auto work) {
            if (progress.done(name)) return true;
            if (stop_after >= 0 && steps >= stop_after) return false;
            const auto t0 = std::chrono::steady_clock::now();
            const long long out = work();
            const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            progress.mark(name);
            ++steps;
            if (!log_path.empty()) {
                std::ofstream log(log_path, std::ios::app);
                log << "{\"step\": \"" << name << "\", \"seconds\": " << sec;
                if (out >= 0)
                    log << ", \"depth_pixels\": " << out << ", \"mpix_per_s\": " << (sec > 0 ? out / sec / 1e6 : 0.0);
                else
                    log << ", \"points\": " << -out;
                log << "}\n";
                if (!log) throw hpm_host::Error(HPM_ERR_IO, "cannot write " + log_path);
            }
            return true;
        };
        auto stopped = [&]() {
            std::cout << "Stopped after " << steps << " steps; --resume continues" << std::endl;
            return 0;
        };
        if (acmm) {
            if (!step("scene", [&] {
                    return hpm_host::RunSceneAcmm(dense_folder, problems, geom_iterations, seed, device);
                }))
                return stopped();
        } else if (!per_problem) {
            if (!step("scene", [&] {
                    return hpm_host::RunScene(dense_folder, problems, planar_prior, geom_iterations, seed, levels,
                                              device, compat);
                }))
                return stopped();
        } else {
            for (size_t p = 0; p < problems.size(); ++p)
                if (!step("A " + std::to_string(problems[p].ref_image_id), [&] {
                        return hpm_host::ProcessProblem(dense_folder, problems[p], false, planar_prior, false,
                                                        seed + p, levels, device, compat);
                    }))
                    return stopped();
            for (int g = 0; g < geom_iterations; ++g)
                for (size_t p = 0; p < problems.size(); ++p)
                    if (!step("G" + std::to_string(g) + " " + std::to_string(problems[p].ref_image_id), [&] {
                            return hpm_host::ProcessProblem(dense_folder, problems[p], true, false, g > 0,
                                                            seed + 1000003ull * (g + 1) + p, levels, device, compat);
                        }))
                        return stopped();
        }
        if (fusion &&
            !step("fusion", [&] {
                const long long n = acmm ? hpm_host::RunFusionAcmm(dense_folder, problems, device)
                                         : hpm_host::RunFusion(dense_folder, problems, geom_iterations > 0, device);
                std::cout << "Fused " << n << " points into " << dense_folder
                          << (acmm ? "/ACMM_NESP/ACMM_NESP_model.ply" : "/HPM/HPM_model.ply") << std::endl;
                return -n;
            }))
            return stopped();
    } catch (const hpm_host::Error &e) {
        std::cerr << "hpm_mvs: " << e.what() << " (status " << e.code << ")" << std::endl;
        return 1;
    }
    return 0;
}
