// Differentiable solving (gb_diff_*): implementation pending.
#include "../../include/ganit_b200.h"
#include "gb_common.cuh"
namespace gb { extern thread_local std::string g_last_error; }
extern "C" {
int gb_diff_create(int, const gb_lp*, const gb_options*, int, int, gb_diff**) { gb::g_last_error = "not built yet"; return GB_ERR_UNSUPPORTED; }
int gb_diff_forward(gb_diff*, const gb_options*, gb_result*, double*, double*) { return GB_ERR_UNSUPPORTED; }
int gb_diff_backward(gb_diff*, const double*, const double*, double*, double*, double*, double*) { return GB_ERR_UNSUPPORTED; }
void gb_diff_destroy(gb_diff*) {}
}
