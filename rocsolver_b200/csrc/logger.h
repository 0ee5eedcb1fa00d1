// logger.h -- multi-level logging (trace, bench and profile logs) of the entry points.
//
// Replaces the reference's logger (library/src/include/rocsolver_logger.hpp:28-70 macros,
// :124-372 class; library/src/common/rocsolver_logger.cpp) behind the same C API
// (rocsolver_log_begin / _end / _set_layer_mode / _set_max_levels / _restore_defaults /
// _write_profile / _flush_profile) and the same environment: ROCSOLVER_LAYER (bit mask:
// 1 trace, 2 bench, 4 profile, 0x10 kernel launches), ROCSOLVER_LEVELS, ROCSOLVER_LOG_PATH and
// ROCSOLVER_LOG_{TRACE,BENCH,PROFILE}_PATH.  Line formats follow the reference's so that its
// tooling reads them:
//   bench   : ./rocsolver-bench -f getrf_strided_batched -r d -m 256 -n 256 --lda 256 ...
//   trace   : ------- ENTER rocsolver_dgetrf_strided_batched trace tree -------
//             rocsolver_getrf_template (m 256, n 256, ...)      (4 spaces per nested level)
//             ------- EXIT rocsolver_dgetrf_strided_batched trace tree -------
//   profile : rocsolver_getrf_template: Calls: 3, Total Time: 12.345 ms
//             (in nested functions: ... ms), kernel launches nested below (with 0x10)
// Profile timing synchronises the handle's stream on exit from each nested step (as the
// reference's does), so profile logging must be off while a stream is being captured.
// With no log session or a zero layer mode every entry point pays one relaxed atomic load.
#pragma once

#include <stdint.h>

#include <initializer_list>
#include <optional>
#include <string>
#include <type_traits>

#include "../../include/rocsolver.h"

namespace rsb {
namespace logging {

constexpr uint32_t TRACE = 1, BENCH = 2, PROFILE = 4, KERNEL = 0x10;

// layer mode of the active session (0 without one)
uint32_t mode();
inline bool enabled() { return (mode() & (TRACE | BENCH | PROFILE)) != 0; }
inline bool kernels() { return enabled() && (mode() & KERNEL) != 0; }

// one "key value" pair of a logged call
struct Arg
{
    const char* key;
    std::string val;
};
template <typename I, typename std::enable_if<std::is_integral<I>::value, int>::type = 0>
inline Arg arg(const char* k, I v)
{
    return Arg{k, std::to_string(v)};
}
inline Arg arg(const char* k, rocblas_operation v)
{
    return Arg{k, v == rocblas_operation_none ? "N"
                  : v == rocblas_operation_transpose ? "T"
                  : v == rocblas_operation_conjugate_transpose ? "C" : "?"};
}
inline Arg arg(const char* k, rocblas_fill v)
{
    return Arg{k, v == rocblas_fill_upper ? "U" : v == rocblas_fill_lower ? "L"
                  : v == rocblas_fill_full ? "F" : "?"};
}

// Logged scope: the constructor logs the entry, the destructor the exit.  top = an exported
// entry point (bench line, trace-tree delimiters, level 0); otherwise a nested step (trace
// line at its level, profile entry).  prec: 's' or 'd' (0 for none).
class Scope
{
public:
    Scope(rocblas_handle h, char prec, const char* name, std::initializer_list<Arg> args,
          bool top);
    ~Scope();
    Scope(const Scope&) = delete;
    Scope& operator=(const Scope&) = delete;

private:
    rocblas_handle handle_;
    bool top_;
    bool active_;
};

// handle of the exported call running on this thread (nullptr outside one): nested steps
// and kernel launches are logged against it
rocblas_handle current();

} // namespace logging
} // namespace rsb

// Log an exported entry point (first statement; `handle` in scope).
#define RSB_LOG_TOP(prec, name, ...)                                                            \
    std::optional<rsb::logging::Scope> _rsb_log_top;                                                \
    if(rsb::logging::enabled())                                                                     \
    _rsb_log_top.emplace(handle, prec, name, std::initializer_list<rsb::logging::Arg>{__VA_ARGS__}, true)

// Log a nested step (a template-level routine) of the current call.
#define RSB_LOG_STEP(name, ...)                                                                 \
    std::optional<rsb::logging::Scope> _rsb_log_step;                                               \
    if(rsb::logging::enabled() && rsb::logging::current())                                              \
    _rsb_log_step.emplace(rsb::logging::current(), 0, name,                                         \
                          std::initializer_list<rsb::logging::Arg>{__VA_ARGS__}, false)

// Log one kernel launch of the current call (layer mode bit 0x10), as a nested step that
// ends with the enclosing block.
#define RSB_LOG_KERNEL(name)                                                                    \
    std::optional<rsb::logging::Scope> _rsb_log_kernel;                                             \
    if(rsb::logging::kernels() && rsb::logging::current())                                              \
    _rsb_log_kernel.emplace(rsb::logging::current(), 0, name, std::initializer_list<rsb::logging::Arg>{}, \
                            false)
