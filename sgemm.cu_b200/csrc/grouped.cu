// grouped.cu — persistent grouped GEMM (under construction).
#include "common.h"

struct sgemm_b200_grouped_plan { int dummy; };

extern "C" int sgemm_b200_grouped_plan_create(sgemm_b200_grouped_plan** plan,
                                              const sgemm_b200_problem* problems, int count,
                                              const char* tuning_json) {
    (void)plan; (void)problems; (void)count; (void)tuning_json;
    return SGEMM_B200_ERR_UNSUPPORTED;
}
extern "C" int sgemm_b200_grouped_plan_launch(sgemm_b200_grouped_plan* plan,
                                              sgemm_b200_stream_t stream, int use_graph) {
    (void)plan; (void)stream; (void)use_graph;
    return SGEMM_B200_ERR_UNSUPPORTED;
}
extern "C" int sgemm_b200_grouped_plan_info(const sgemm_b200_grouped_plan* plan, int* tiles,
                                            int* work_items, int* grid_ctas) {
    (void)plan; (void)tiles; (void)work_items; (void)grid_ctas;
    return SGEMM_B200_ERR_UNSUPPORTED;
}
extern "C" void sgemm_b200_grouped_plan_destroy(sgemm_b200_grouped_plan* plan) { (void)plan; }
extern "C" int sgemm_b200_grouped(const sgemm_b200_problem* problems, int count,
                                  sgemm_b200_stream_t stream) {
    (void)problems; (void)count; (void)stream;
    return SGEMM_B200_ERR_UNSUPPORTED;
}
extern "C" int sgemm_b200_autotune_grouped(const sgemm_b200_problem* problems, int count,
                                           const char* json_path) {
    (void)problems; (void)count; (void)json_path;
    return SGEMM_B200_ERR_UNSUPPORTED;
}
