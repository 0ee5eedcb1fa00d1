// bounds.cpp -- host side of the bounds-checked build (common.cuh, RSB_BOUNDS_CHECK): every
// translation unit registers a query of its device record; rocsolver_b200_bounds_check sums
// them.  In the normal build the entry point reports that no checks are compiled in.
#include <mutex>
#include <vector>

#include "../../include/rocsolver.h"

namespace rsb {
namespace bounds {
typedef void (*QueryFn)(int* out4);
namespace {
std::mutex& mu()
{
    static std::mutex m;
    return m;
}
std::vector<QueryFn>& fns()
{
    static std::vector<QueryFn> v;
    return v;
}
} // namespace
void register_query(QueryFn f)
{
    std::lock_guard<std::mutex> lk(mu());
    fns().push_back(f);
}
} // namespace bounds
} // namespace rsb

extern "C" rocblas_status rocsolver_b200_bounds_check(rocblas_int* result)
{
#ifdef RSB_BOUNDS_CHECK
    if(!result)
        return rocblas_status_invalid_pointer;
    result[0] = result[1] = result[2] = result[3] = 0;
    std::lock_guard<std::mutex> lk(rsb::bounds::mu());
    for(rsb::bounds::QueryFn f : rsb::bounds::fns())
        f(result);
    return rocblas_status_success;
#else
    (void)result;
    return rocblas_status_not_implemented;
#endif
}
