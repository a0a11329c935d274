/*
 * C entry point of the fusion checkers: runs the reference's own RunFusion on
 * a dense folder, HPM-MVS/main.cpp:502-633 in oracle/_ref/libfusion_ref.so,
 * the ACMM+NESP variant's (ACMM+NESP/windows/main.cpp:154-297) in
 * oracle/_ref/libfusion_acmm_ref.so (both compiled from the reference tree by
 * oracle/Makefile).
 *
 * TEST INFRASTRUCTURE ONLY.
 */
#include "fusion_stub.h"

void RunFusion(std::string &dense_folder, const std::vector<Problem> &problems, bool geom_consistency);

/* problems as in hpm_run_scene: ref_ids[n], src_counts[n], src_ids[n][32];
 * writes the PLY as the reference does (dense_folder/HPM/HPM_model.ply, or
 * dense_folder/ACMM_NESP/ACMM_NESP_model.ply for the variant).  The
 * reference's progress lines go nowhere. */
extern "C" int ref_run_fusion(const char *dense_folder, int n, const int *ref_ids, const int *src_counts,
                              const int *src_ids, int geom_consistency)
{
    if (!dense_folder || n < 1 || !ref_ids || !src_counts || !src_ids) return -1;
    std::vector<Problem> problems(n);
    for (int i = 0; i < n; ++i) {
        problems[i].ref_image_id = ref_ids[i];
        problems[i].src_image_ids.assign(src_ids + 32 * i, src_ids + 32 * i + src_counts[i]);
    }
    std::string folder(dense_folder);
    std::streambuf *saved = std::cout.rdbuf(nullptr);
    RunFusion(folder, problems, geom_consistency != 0);
    std::cout.rdbuf(saved);
    return 0;
}
