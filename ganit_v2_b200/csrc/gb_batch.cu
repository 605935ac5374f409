// Batched solving (gb_batch_*): implementation pending.
#include "../../include/ganit_b200.h"
#include "gb_common.cuh"
namespace gb { extern thread_local std::string g_last_error; }
extern "C" {
int gb_batch_create(int, const gb_lp*, const gb_options*, gb_batch**) { gb::g_last_error = "not built yet"; return GB_ERR_UNSUPPORTED; }
int gb_batch_solve(gb_batch*, const gb_options*, gb_result*) { return GB_ERR_UNSUPPORTED; }
int gb_batch_get_solution(gb_batch*, int, double*, double*) { return GB_ERR_UNSUPPORTED; }
int gb_batch_schedule(gb_batch*, int*, int*, int*) { return GB_ERR_UNSUPPORTED; }
void gb_batch_destroy(gb_batch*) {}
}
